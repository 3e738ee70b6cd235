// Drop-in shims with the reference's signatures (see include/nspb_compat.h).
#include "../../include/nspb_compat.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

static nspb_csr_in as_in(const sfCSR *m, int nrows, int ncols) {
  nspb_csr_in d;
  std::memset(&d, 0, sizeof(d));
  d.nrows = nrows;
  d.ncols = ncols;
  d.nnz = m->nnz;
  d.rowptr = m->d_rpt;
  d.col = m->d_col;
  d.val = m->d_val;
  d.val_type = NSPB_F64;
  return d;
}

extern "C" int nspb_nsp_spgemm_kernel_hash(sfCSR *a, sfCSR *b, sfCSR *c) {
  if (!a || !b || !c) return NSPB_ERR_INVALID;
  if (a->M > 0x7fffffffu || a->N > 0x7fffffffu || b->M > 0x7fffffffu || b->N > 0x7fffffffu)
    return NSPB_ERR_INVALID;
  // a->N is the number of B rows; the reference never reads it, so take it
  // from b->M when a->N is unset
  const int inner = b->M ? (int)b->M : (int)a->N;
  nspb_csr_in A = as_in(a, (int)a->M, inner);
  nspb_csr_in B = as_in(b, inner, (int)b->N);
  nspb_csr_out C;
  std::memset(&C, 0, sizeof(C));
  nspb_opts o;
  nspb_default_opts(&o);
  int st = nspb_spgemm(&A, &B, &C, &o, nullptr);
  if (st) return st;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    return NSPB_ERR_CUDA;
  }
  c->M = a->M;
  c->N = b->N;
  c->nnz = (int)C.nnz;
  c->d_rpt = C.rowptr;
  c->d_col = C.col;
  c->d_val = C.val;
  return NSPB_OK;
}

void nsp_spgemm_kernel_hash(sfCSR *a, sfCSR *b, sfCSR *c) {
  const int st = nspb_nsp_spgemm_kernel_hash(a, b, c);
  if (st) {
    std::fprintf(stderr, "nsp_spgemm_kernel_hash: %s (cuda error %d)\n", nspb_strerror(st),
                 nspb_last_cuda_error());
    std::exit(EXIT_FAILURE);
  }
}

CSR *nsparseMGPU_version0(CSR *Alocal, CSR *Pfull, csrlocinfo *Plocal, double &loc_time) {
  (void)Plocal;
  if (!Alocal || !Pfull || !Alocal->on_the_device || !Pfull->on_the_device) {
    std::fprintf(stderr, "nsparseMGPU_version0: operands must be on the device\n");
    std::exit(EXIT_FAILURE);
  }
  sfCSR a, p, c;
  std::memset(&a, 0, sizeof(a));
  std::memset(&p, 0, sizeof(p));
  std::memset(&c, 0, sizeof(c));
  a.M = (unsigned)Alocal->n;
  a.N = (unsigned)Alocal->m;
  a.nnz = (int)Alocal->nnz;
  a.d_rpt = Alocal->row;
  a.d_col = Alocal->col;
  a.d_val = Alocal->val;
  p.M = (unsigned)Pfull->n;
  p.N = (unsigned)Pfull->m;
  p.nnz = (int)Pfull->nnz;
  p.d_rpt = Pfull->row;
  p.d_col = Pfull->col;
  p.d_val = Pfull->val;

  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  nsp_spgemm_kernel_hash(&a, &p, &c);
  cudaDeviceSynchronize();
  loc_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  CSR *C = static_cast<CSR *>(std::calloc(1, sizeof(CSR)));
  void **descr = static_cast<void **>(std::calloc(1, sizeof(void *)));
  if (!C || !descr) {
    std::fprintf(stderr, "nsparseMGPU_version0: host allocation failed\n");
    std::exit(EXIT_FAILURE);
  }
  C->nnz = (stype)c.nnz;
  C->n = (stype)c.M;
  C->m = (gstype)c.N;
  C->shrinked_m = (stype)c.N;
  C->full_n = Alocal->full_n;
  C->full_m = (gstype)c.N;
  C->on_the_device = true;
  C->row_shift = Alocal->row_shift;
  C->row = c.d_rpt;
  C->col = c.d_col;
  C->val = c.d_val;
  C->descr = descr;
  C->halo.init = false;
  C->rows_to_get = nullptr;
  return C;
}

CSR *nsparseMGPU_version1(handles *h, CSR *Alocal, CSR *Plocal, double &loc_time) {
  (void)h;
  csrlocinfo info;
  info.fr = 0;
  info.lr = Plocal ? (int)Plocal->n : 0;
  info.row = Plocal ? Plocal->row : nullptr;
  info.col = nullptr;
  info.val = Plocal ? Plocal->val : nullptr;
  return nsparseMGPU_version0(Alocal, Plocal, &info, loc_time);
}
