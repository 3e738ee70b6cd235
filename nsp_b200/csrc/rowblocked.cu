// Row-blocked product for a C larger than a device-memory budget.
//
// The reference forms the product of a row block against the B rows that
// block references by compressing A's column space (get_shrinked_matrix,
// src/spspmpi.cu:106-182, with getmct src/getmct.cu:135-220 and the binary
// search remap src/spspmpi.cu:58-104) before its local product
// (src/spspmpi.cu:906-935). Here the same remap drives an out-of-core product
// on one GPU: C's row counts come from one symbolic pass over all rows; rows
// are cut into blocks whose C fits the budget; per block the referenced B rows
// are gathered into a compact B (getmct + row gather), A's block columns are
// remapped into it (shrink), the block's numeric step runs, and the block of
// C is copied to the caller's host arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "remap.h"
#include "spgemm_host.h"

namespace nspb {

__global__ void k_rebase(const int *__restrict__ in, long long first, long long n,
                         int *__restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[first + i] - in[first];
}

__global__ void k_gather_len(const int *__restrict__ brpt, const int *__restrict__ rows, int m,
                             int *__restrict__ len) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
    len[j] = brpt[rows[j] + 1] - brpt[rows[j]];
}

// One warp per gathered row copies its entries.
__global__ void k_gather_rows(const int *__restrict__ brpt, const int *__restrict__ bcol,
                              const double *__restrict__ bval, const int *__restrict__ rows,
                              int m, const int *__restrict__ grpt, int *__restrict__ gcol,
                              double *__restrict__ gval) {
  const int lane = threadIdx.x & 31;
  for (long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < m;
       j += ((long long)gridDim.x * blockDim.x) >> 5) {
    const int s0 = brpt[rows[j]], s1 = brpt[rows[j] + 1];
    const int d = grpt[j];
    for (int e = s0 + lane; e < s1; e += 32) {
      gcol[d + e - s0] = bcol[e];
      gval[d + e - s0] = bval[e];
    }
  }
}

static int gcap(long long n) {
  const long long g = (n + 255) / 256, cap = (long long)dev_info().sms * 16;
  return (int)std::max<long long>(1, std::min(g, cap));
}

}  // namespace nspb

using namespace nspb;

extern "C" int nspb_spgemm_rowblocked(const nspb_csr_in *A, const nspb_csr_in *B,
                                      int64_t budget_bytes, int32_t *h_rowptr, int32_t *h_col,
                                      double *h_val, int64_t h_capacity, int64_t *nnz_out,
                                      int32_t *nblocks_out, const nspb_opts *opts) {
  if (!A || !B || !h_rowptr || !nnz_out || !nblocks_out || budget_bytes <= 0)
    return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  if (o.precision != NSPB_PREC_FP64) return NSPB_ERR_UNSUPPORTED;
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  const int n = A->nrows;
  *nblocks_out = 0;
  // 1. row counts of all of C (device row pointer, then host copy)
  int *d_crpt = nullptr;
  int st = scratch_alloc(reinterpret_cast<void **>(&d_crpt), 4 * ((size_t)n + 1), s);
  if (st) return st;
  nspb_csr_out Cfull;
  std::memset(&Cfull, 0, sizeof(Cfull));
  Cfull.rowptr = d_crpt;
  st = nspb_spgemm_symbolic(A, B, &Cfull, &o, nullptr);
  std::vector<int> arpt((size_t)n + 1, 0);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(h_rowptr, d_crpt, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n > 0)
      e = cudaMemcpyAsync(arpt.data(), A->rowptr, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      g_last_cuda = (int)e;
      st = NSPB_ERR_CUDA;
    }
  }
  if (st) {
    scratch_free(d_crpt, s);
    return st;
  }
  *nnz_out = Cfull.nnz;
  if (Cfull.nnz > h_capacity || (Cfull.nnz > 0 && (!h_col || !h_val))) {
    scratch_free(d_crpt, s);
    return NSPB_ERR_CAPACITY;
  }
  // 2. blocks of rows whose C (12 B per entry + 4 B per row) fits the budget
  std::vector<int> cut{0};
  {
    long long bytes = 0;
    for (int i = 0; i < n; ++i) {
      const long long rb = 12LL * (h_rowptr[i + 1] - h_rowptr[i]) + 4;
      if (bytes + rb > budget_bytes && i > cut.back()) {
        cut.push_back(i);
        bytes = 0;
      }
      bytes += rb;
    }
    cut.push_back(n);
  }
  // 3. per block: remap, gather, numeric step, copy out
  for (size_t b = 0; b + 1 < cut.size() && !st; ++b) {
    const int r0 = cut[b], r1 = cut[b + 1];
    const long long a_lo = arpt[r0], a_len = (long long)arpt[r1] - a_lo;
    const long long c_lo = h_rowptr[r0], c_len = (long long)h_rowptr[r1] - c_lo;
    const int nr = r1 - r0;
    // scratch: needed columns, shrunk A columns, rebased row pointers, lengths
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    size_t off = 0;
    const size_t o_cols = off; off = al(off + 4 * (size_t)std::max<long long>(a_len, 1));
    const size_t o_acol = off; off = al(off + 4 * (size_t)std::max<long long>(a_len, 1));
    const size_t o_arp = off; off = al(off + 4 * ((size_t)nr + 1));
    const size_t o_crp = off; off = al(off + 4 * ((size_t)nr + 1));
    const size_t o_len = off; off = al(off + 4 * ((size_t)std::max<long long>(a_len, 1) + 1));
    const size_t o_hdr = off; off = al(off + 128);
    const size_t o_tiles = off; off = al(off + 8 * (size_t)scan_tiles((int)std::max<long long>(a_len, 1)));
    char *ws = nullptr;
    if ((st = scratch_alloc(reinterpret_cast<void **>(&ws), off, s))) break;
    int *cols = reinterpret_cast<int *>(ws + o_cols);
    int *acol = reinterpret_cast<int *>(ws + o_acol);
    int *barp = reinterpret_cast<int *>(ws + o_arp);
    int *bcrp = reinterpret_cast<int *>(ws + o_crp);
    int *len = reinterpret_cast<int *>(ws + o_len);
    int64_t m = 0;
    int *gcol = nullptr, *grpt = nullptr, *ccol = nullptr;
    double *gval = nullptr, *cval = nullptr;
    cudaError_t e = cudaMemsetAsync(ws + o_hdr, 0, off - o_hdr, s);
    if (e == cudaSuccess) {
      st = getmct_dev(A->col + a_lo, a_len, 1, 0, cols, &m, s);
    } else {
      st = NSPB_ERR_CUDA;
    }
    long long g_nnz = 0;
    if (!st && m > 0) {
      // gathered B: row lengths -> row pointer (single-pass scan) -> entries
      k_gather_len<<<gcap(m), 256, 0, s>>>(B->rowptr, cols, (int)m, len);
      long long *tot = reinterpret_cast<long long *>(ws + o_hdr);
      int *ctr = reinterpret_cast<int *>(ws + o_hdr + 8);
      int *errw = reinterpret_cast<int *>(ws + o_hdr + 12);
      int *hist = reinterpret_cast<int *>(ws + o_hdr + 16);
      st = alloc_out(reinterpret_cast<void **>(&grpt), 4 * ((size_t)m + 1));
      if (!st) {
        e = launch_scan(len, (int)m, grpt, tot, reinterpret_cast<unsigned long long *>(ws + o_tiles),
                        ctr, bin_limits(0, 0), hist, errw, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&g_nnz, tot, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = NSPB_ERR_CUDA;
      }
      if (!st) st = alloc_out(reinterpret_cast<void **>(&gcol), 4 * (size_t)std::max<long long>(g_nnz, 1));
      if (!st) st = alloc_out(reinterpret_cast<void **>(&gval), 8 * (size_t)std::max<long long>(g_nnz, 1));
      if (!st) {
        k_gather_rows<<<gcap(32 * m), 256, 0, s>>>(B->rowptr, B->col,
                                                   static_cast<const double *>(B->val), cols,
                                                   (int)m, grpt, gcol, gval);
        if (a_len) st = shrink_col_dev(A->col + a_lo, a_len, cols, m, acol, s);
      }
    }
    if (!st) {
      k_rebase<<<gcap(nr + 1), 256, 0, s>>>(A->rowptr, r0, nr, barp);
      k_rebase<<<gcap(nr + 1), 256, 0, s>>>(d_crpt, r0, nr, bcrp);
      if ((e = cudaGetLastError()) != cudaSuccess) st = NSPB_ERR_CUDA;
    }
    if (!st && c_len > 0) {
      st = alloc_out(reinterpret_cast<void **>(&ccol), 4 * (size_t)c_len);
      if (!st) st = alloc_out(reinterpret_cast<void **>(&cval), 8 * (size_t)c_len);
      if (!st) {
        const double *aval = static_cast<const double *>(A->val);
        nspb_csr_in Ab = {nr, (int32_t)m, a_len, barp, acol, aval + a_lo, NSPB_F64, 0};
        nspb_csr_in Bb = {(int32_t)m, B->ncols, g_nnz, grpt, gcol, gval, NSPB_F64, 0};
        nspb_csr_out Cb = {nr, B->ncols, c_len, bcrp, ccol, cval, c_len};
        st = nspb_spgemm_numeric(&Ab, &Bb, &Cb, &o, nullptr);
      }
      if (!st) {
        e = cudaMemcpyAsync(h_col + c_lo, ccol, 4 * (size_t)c_len, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(h_val + c_lo, cval, 8 * (size_t)c_len, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = NSPB_ERR_CUDA;
      }
    }
    if (st == NSPB_ERR_CUDA) {
      g_last_cuda = (int)(e != cudaSuccess ? e : cudaGetLastError());
      cudaGetLastError();
    }
    cudaStreamSynchronize(s);
    scratch_free(ws, s);
    cudaFree(grpt);
    cudaFree(gcol);
    cudaFree(gval);
    cudaFree(ccol);
    cudaFree(cval);
    *nblocks_out += 1;
  }
  scratch_free(d_crpt, s);
  return st;
}
