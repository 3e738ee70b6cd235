// A host program written against the reference's own interface, the way its
// driver uses it: CSR operands on the device built like CSRm::init
// (src/CSR.cu:28-120, a cuSPARSE descriptor included), the product through
// nsparseMGPU_version1 (src/spspmpi.h:31, called from src/main.cu:223) and
// through nsp_spgemm_kernel_hash on sfCSR (nsp/inc/nsp.h:105), and C
// released the way CSRm::free does (src/CSR.cu:572-620): cudaFree of its
// arrays, cusparseDestroyMatDescr(*descr), free(descr), free(C).
// It includes only include/nspb_compat.h and links libnspb.so; the test that
// builds it compares the products it writes with the oracle.
//
// usage: caller <A file> <B file> <out prefix>
//   input file:  int32 nrows, ncols, nnz; int32 rowptr[nrows+1]; int32 col[nnz];
//                fp64 val[nnz]
//   writes <out prefix>.v1 (nsparseMGPU_version1) and <out prefix>.kh
//   (nsp_spgemm_kernel_hash) in the same layout, and prints loc_time and the
//   status of cusparseDestroyMatDescr on each returned descriptor.
#include <cuda_runtime.h>
#include <cusparse.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "nspb_compat.h"

namespace {

struct HostCsr {
  int n = 0, m = 0, nnz = 0;
  std::vector<int> rp, col;
  std::vector<double> val;
};

bool read_csr(const char *path, HostCsr &h) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  int hdr[3];
  bool ok = std::fread(hdr, sizeof(int), 3, f) == 3;
  if (ok) {
    h.n = hdr[0];
    h.m = hdr[1];
    h.nnz = hdr[2];
    h.rp.resize((size_t)h.n + 1);
    h.col.resize((size_t)h.nnz);
    h.val.resize((size_t)h.nnz);
    ok = std::fread(h.rp.data(), sizeof(int), h.rp.size(), f) == h.rp.size() &&
         std::fread(h.col.data(), sizeof(int), h.col.size(), f) == h.col.size() &&
         std::fread(h.val.data(), sizeof(double), h.val.size(), f) == h.val.size();
  }
  std::fclose(f);
  return ok;
}

bool write_csr(const char *path, int n, int m, int nnz, const int *d_rp, const int *d_col,
               const double *d_val) {
  std::vector<int> rp((size_t)n + 1), col((size_t)nnz);
  std::vector<double> val((size_t)nnz);
  if (cudaMemcpy(rp.data(), d_rp, rp.size() * sizeof(int), cudaMemcpyDeviceToHost) ||
      (nnz && cudaMemcpy(col.data(), d_col, col.size() * sizeof(int), cudaMemcpyDeviceToHost)) ||
      (nnz && cudaMemcpy(val.data(), d_val, val.size() * sizeof(double), cudaMemcpyDeviceToHost)))
    return false;
  FILE *f = std::fopen(path, "wb");
  if (!f) return false;
  const int hdr[3] = {n, m, nnz};
  std::fwrite(hdr, sizeof(int), 3, f);
  std::fwrite(rp.data(), sizeof(int), rp.size(), f);
  std::fwrite(col.data(), sizeof(int), col.size(), f);
  std::fwrite(val.data(), sizeof(double), val.size(), f);
  std::fclose(f);
  return true;
}

template <typename T>
T *upload(const std::vector<T> &h) {
  T *d = nullptr;
  if (cudaMalloc(&d, (h.size() ? h.size() : 1) * sizeof(T)) != cudaSuccess) return nullptr;
  if (!h.empty()) cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}

// A device CSR as CSRm::init + copyToDevice leave it.
CSR *make_device_csr(const HostCsr &h) {
  CSR *A = static_cast<CSR *>(std::calloc(1, sizeof(CSR)));
  A->nnz = (stype)h.nnz;
  A->n = (stype)h.n;
  A->m = (gstype)h.m;
  A->shrinked_m = (stype)h.m;
  A->full_n = (gstype)h.n;
  A->full_m = (gstype)h.m;
  A->on_the_device = true;
  A->row = upload(h.rp);
  A->col = upload(h.col);
  A->val = upload(h.val);
  cusparseMatDescr_t *descr = static_cast<cusparseMatDescr_t *>(std::malloc(sizeof(cusparseMatDescr_t)));
  cusparseCreateMatDescr(descr);
  cusparseSetMatIndexBase(*descr, CUSPARSE_INDEX_BASE_ZERO);
  cusparseSetMatType(*descr, CUSPARSE_MATRIX_TYPE_GENERAL);
  A->descr = reinterpret_cast<void **>(descr);
  return A;
}

// CSRm::free for a device CSR; returns the status of cusparseDestroyMatDescr.
int free_device_csr(CSR *A) {
  cudaFree(A->val);
  cudaFree(A->col);
  cudaFree(A->row);
  if (A->shrinked_col) cudaFree(A->shrinked_col);
  const int st = (int)cusparseDestroyMatDescr(*reinterpret_cast<cusparseMatDescr_t *>(A->descr));
  std::free(A->descr);
  std::free(A);
  return st;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s <A file> <B file> <out prefix>\n", argv[0]);
    return 2;
  }
  HostCsr ha, hb;
  if (!read_csr(argv[1], ha) || !read_csr(argv[2], hb)) {
    std::fprintf(stderr, "cannot read the operands\n");
    return 2;
  }
  CSR *A = make_device_csr(ha);
  CSR *B = make_device_csr(hb);
  std::string prefix(argv[3]);

  // the driver's call (src/main.cu:223): one GPU, no MPI
  double loc_time = -1.0;
  CSR *C = nsparseMGPU_version1(nullptr, A, B, loc_time);
  if (C->n != A->n || C->m != B->m || !C->on_the_device || C->full_n != A->full_n ||
      C->row_shift != A->row_shift) {
    std::fprintf(stderr, "nsparseMGPU_version1: unexpected CSR fields\n");
    return 1;
  }
  if (!write_csr((prefix + ".v1").c_str(), (int)C->n, (int)C->m, (int)C->nnz, C->row, C->col,
                 C->val))
    return 1;
  const int st_v1 = free_device_csr(C);

  // the kernel-level entry on sfCSR
  sfCSR a, b, c;
  std::memset(&a, 0, sizeof(a));
  std::memset(&b, 0, sizeof(b));
  std::memset(&c, 0, sizeof(c));
  a.M = (unsigned)ha.n;
  a.N = (unsigned)ha.m;
  a.nnz = ha.nnz;
  a.d_rpt = A->row;
  a.d_col = A->col;
  a.d_val = A->val;
  b.M = (unsigned)hb.n;
  b.N = (unsigned)hb.m;
  b.nnz = hb.nnz;
  b.d_rpt = B->row;
  b.d_col = B->col;
  b.d_val = B->val;
  nsp_spgemm_kernel_hash(&a, &b, &c);
  if (c.M != a.M || c.N != b.N) {
    std::fprintf(stderr, "nsp_spgemm_kernel_hash: unexpected sfCSR fields\n");
    return 1;
  }
  if (!write_csr((prefix + ".kh").c_str(), (int)c.M, (int)c.N, c.nnz, c.d_rpt, c.d_col, c.d_val))
    return 1;
  cudaFree(c.d_rpt);
  cudaFree(c.d_col);
  cudaFree(c.d_val);
  const int st_a = free_device_csr(A);
  const int st_b = free_device_csr(B);
  std::printf("loc_time %.9f destroy_descr_C %d destroy_descr_A %d destroy_descr_B %d\n", loc_time,
              st_v1, st_a, st_b);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}
