// CSR transpose and the smoothed-aggregation steps of the AMG Galerkin driver
// (R = P^T, A_c = R (A P), P = P_tent - w D^-1 A P_tent), on one stream.
//
// Reference counterparts: CSRm::T (src/CSR.cu:738-785, cuSPARSE csr2csc),
// CSRm::diag / _getDiagonal (src/CSR.cu:1389-1418). The products go through
// this library's own CSR product.
//
// The transpose is a stable LSD radix sort of A's entries by column: entries
// enter in row order, so every transposed row lists its rows ascending (what
// csr2csc returns) and duplicates keep their order; 8 bits per pass, tiles of
// 4096 entries, each pass one histogram kernel, one scan and one scatter
// kernel whose in-tile ranks come from warp match masks (so the scatter is
// stable without a sort inside the tile).
#include "common.cuh"
#include "internal.h"
#include "spgemm_host.h"

#include <algorithm>
#include <vector>

namespace nspb {

constexpr int kRadixThreads = 256;
constexpr int kRadixPer = 16;
constexpr int kRadixTile = kRadixThreads * kRadixPer;
constexpr int kRadixBins = 256;
constexpr int kRadixWarps = kRadixThreads / 32;

// rows[e] = i for every entry e of row i (one warp per row)
__global__ void k_expand_rows(const int *__restrict__ rpt, int n, int *__restrict__ rows) {
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = w0; i < n; i += nw)
    for (int e = rpt[i] + lane; e < rpt[i + 1]; e += 32) rows[e] = i;
}

// entries per column; a column outside [0, m) raises ERR_CAPACITY
__global__ void k_col_count(const int *__restrict__ col, long long nnz, int m,
                            int *__restrict__ counts, int *__restrict__ err) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    const int c = col[e];
    if ((unsigned)c < (unsigned)m) atomicAdd(counts + c, 1);
    else atomicOr(err, ERR_CAPACITY);
  }
}

// digit histogram of one tile, stored digit-major: hist[d * ntiles + tile]
__global__ void __launch_bounds__(kRadixThreads)
    k_radix_hist(const int *__restrict__ keys, long long nnz, int shift, int ntiles,
                 int *__restrict__ hist) {
  __shared__ int h[kRadixBins];
  const int tile = blockIdx.x;
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)tile * kRadixTile;
#pragma unroll 4
  for (int i = 0; i < kRadixPer; ++i) {
    const long long e = base + i * kRadixThreads + threadIdx.x;
    if (e < nnz) atomicAdd(&h[(keys[e] >> shift) & (kRadixBins - 1)], 1);
  }
  __syncthreads();
  hist[(long long)threadIdx.x * ntiles + tile] = h[threadIdx.x];
}

// Stable scatter of one tile: element e goes to off[d][tile] + (elements of
// digit d before it in the tile). Chunks of 256 elements in order; inside a
// chunk, lanes of a warp with the same digit are ranked by the match mask and
// warps by the per-warp digit counts.
template <typename VT>
__global__ void __launch_bounds__(kRadixThreads)
    k_radix_scatter(const int *__restrict__ keys_in, const int *__restrict__ rows_in,
                    const VT *__restrict__ vals_in, long long nnz, int shift, int ntiles,
                    const int *__restrict__ off, int *__restrict__ keys_out,
                    int *__restrict__ rows_out, VT *__restrict__ vals_out) {
  __shared__ int wcnt[kRadixWarps][kRadixBins];
  __shared__ int run[kRadixBins];
  const int tile = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int w = 0; w < kRadixWarps; ++w) wcnt[w][threadIdx.x] = 0;
  run[threadIdx.x] = off[(long long)threadIdx.x * ntiles + tile];
  __syncthreads();
  const long long base = (long long)tile * kRadixTile;
  for (int i = 0; i < kRadixPer; ++i) {
    const long long e = base + i * kRadixThreads + threadIdx.x;
    const bool valid = e < nnz;
    int key = 0, d = kRadixBins;  // kRadixBins: no element (never indexes)
    if (valid) {
      key = keys_in[e];
      d = (key >> shift) & (kRadixBins - 1);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    int pos = 0;
    if (valid) {
      pos = run[d] + rank;
      for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
    }
    __syncthreads();  // every thread has read run[] and wcnt[]
    int s = 0;
    for (int w = 0; w < kRadixWarps; ++w) {
      s += wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = 0;
    }
    run[threadIdx.x] += s;
    if (valid) {
      if (keys_out) keys_out[pos] = key;
      rows_out[pos] = rows_in[e];
      vals_out[pos] = vals_in[e];
    }
    __syncthreads();
  }
}

// D[i] = a_ii (the last diagonal entry of the row, as _getDiagonal keeps);
// a row without one raises ERR_CAPACITY and gets 0.
__global__ void k_diag(const int *__restrict__ rpt, const int *__restrict__ col,
                       const double *__restrict__ val, int n, double *__restrict__ D,
                       int *__restrict__ err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    bool found = false;
    for (int e = rpt[i]; e < rpt[i + 1]; ++e) {
      if (col[e] == i) {
        d = val[e];
        found = true;
      }
    }
    if (!found) atomicOr(err, ERR_CAPACITY);
    D[i] = d;
  }
}

// P(i,:) = -w AP(i,:) / D[i], then P_tent(i,:) added at its columns (which
// the pattern of A P_tent holds when a_ii is stored). One warp per row; the
// P_tent entries of a row are added by one lane in order (duplicates sum in
// their stored order). A P_tent column missing from the row raises
// ERR_CAPACITY.
__global__ void k_sa_smooth(const int *__restrict__ prpt, const int *__restrict__ pcol,
                            double *__restrict__ pval, const int *__restrict__ trpt,
                            const int *__restrict__ tcol, const double *__restrict__ tval,
                            const double *__restrict__ D, double omega, int n,
                            int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = w0; i < n; i += nw) {
    const int p0 = prpt[i], p1 = prpt[i + 1];
    const double d = D[i];
    for (int e = p0 + lane; e < p1; e += 32) pval[e] = __ddiv_rn(__dmul_rn(-omega, pval[e]), d);
    __syncwarp();
    if (lane == 0) {
      for (int t = trpt[i]; t < trpt[i + 1]; ++t) {
        const int c = tcol[t];
        int lo = p0, hi = p1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (pcol[mid] < c) lo = mid + 1; else hi = mid;
        }
        if (lo < p1 && pcol[lo] == c) pval[lo] = __dadd_rn(pval[lo], tval[t]);
        else atomicOr(err, ERR_CAPACITY);
      }
    }
    __syncwarp();
  }
}

namespace {

int grid_for(long long items, int threads) {
  const long long cap = (long long)dev_info().sms * 16;
  const long long need = (items + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min(need, cap));
}

// Scratch of one call from the library's stream-ordered pool.
struct Scratch {
  cudaStream_t s;
  std::vector<void *> blocks;
  explicit Scratch(cudaStream_t st) : s(st) {}
  ~Scratch() {
    for (void *p : blocks) scratch_free(p, s);
  }
  template <typename T>
  int get(T **p, size_t count) {
    void *q = nullptr;
    const int st = scratch_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), s);
    if (st) return st;
    blocks.push_back(q);
    *p = static_cast<T *>(q);
    return NSPB_OK;
  }
};

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return NSPB_OK;
  g_last_cuda = (int)e;
  cudaGetLastError();
  return NSPB_ERR_CUDA;
}

// Exclusive scan of in[0..n) into out[0..n] (out[n] = total) with the
// product's single-pass scan kernel.
int scan_into(const int *in, int n, int *out, Scratch &ws, cudaStream_t s) {
  if (n <= 0) return cuda_status(cudaMemsetAsync(out, 0, sizeof(int), s));
  struct Ctr {
    long long total;
    int tile_ctr, err;
    int num_counts[16];
  };
  Ctr *ctr = nullptr;
  unsigned long long *tiles = nullptr;
  int st;
  if ((st = ws.get(&ctr, 1)) || (st = ws.get(&tiles, (size_t)scan_tiles(n)))) return st;
  cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(Ctr), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(tiles, 0, (size_t)scan_tiles(n) * sizeof(unsigned long long), s);
  if (e == cudaSuccess)
    e = launch_scan(in, n, out, &ctr->total, tiles, &ctr->tile_ctr, bin_limits(0, 0),
                    ctr->num_counts, &ctr->err, s);
  return cuda_status(e);
}

template <typename VT>
int transpose_t(const nspb_csr_in *A, int32_t *trpt, int32_t *tcol, VT *tval, int *err,
                cudaStream_t s) {
  const int n = A->nrows, m = A->ncols;
  const long long nnz = A->nnz;
  Scratch ws(s);
  int st;
  int *counts = nullptr;
  if ((st = ws.get(&counts, (size_t)m + 1))) return st;
  if ((st = cuda_status(cudaMemsetAsync(counts, 0, ((size_t)m + 1) * sizeof(int), s)))) return st;
  if (nnz > 0) {
    k_col_count<<<grid_for(nnz, 256), 256, 0, s>>>(A->col, nnz, m, counts, err);
    if ((st = cuda_status(cudaGetLastError()))) return st;
  }
  if ((st = scan_into(counts, m, trpt, ws, s))) return st;
  if (nnz == 0) return NSPB_OK;
  int *rows = nullptr;
  if ((st = ws.get(&rows, (size_t)nnz))) return st;
  k_expand_rows<<<grid_for((long long)n * 32, 256), 256, 0, s>>>(A->rowptr, n, rows);
  if ((st = cuda_status(cudaGetLastError()))) return st;
  int bits = 0;
  while (bits < 31 && ((long long)(m - 1) >> bits) > 0) ++bits;
  const int passes = std::max(1, (bits + 7) / 8);
  const int ntiles = (int)((nnz + kRadixTile - 1) / kRadixTile);
  int *hist = nullptr, *off = nullptr;
  if ((st = ws.get(&hist, (size_t)kRadixBins * ntiles)) ||
      (st = ws.get(&off, (size_t)kRadixBins * ntiles + 1)))
    return st;
  int *kbuf[2] = {nullptr, nullptr}, *rbuf[2] = {nullptr, nullptr};
  VT *vbuf[2] = {nullptr, nullptr};
  for (int b = 0; b < (passes > 1 ? 2 : 0); ++b)
    if ((st = ws.get(&kbuf[b], (size_t)nnz)) || (st = ws.get(&rbuf[b], (size_t)nnz)) ||
        (st = ws.get(&vbuf[b], (size_t)nnz)))
      return st;
  const int *kin = A->col, *rin = rows;
  const VT *vin = static_cast<const VT *>(A->val);
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    const bool last = p == passes - 1;
    int *kout = last ? nullptr : kbuf[p & 1];
    int *rout = last ? tcol : rbuf[p & 1];
    VT *vout = last ? tval : vbuf[p & 1];
    k_radix_hist<<<ntiles, kRadixThreads, 0, s>>>(kin, nnz, shift, ntiles, hist);
    if ((st = cuda_status(cudaGetLastError()))) return st;
    if ((st = scan_into(hist, kRadixBins * ntiles, off, ws, s))) return st;
    k_radix_scatter<VT><<<ntiles, kRadixThreads, 0, s>>>(kin, rin, vin, nnz, shift, ntiles, off,
                                                         kout, rout, vout);
    if ((st = cuda_status(cudaGetLastError()))) return st;
    kin = kout;
    rin = rout;
    vin = vout;
  }
  return NSPB_OK;
}

// Device error word of a call, read back once at its end.
struct ErrWord {
  int *d = nullptr;
  int read(cudaStream_t s, int *h) {
    HostStage *hs = host_stage();
    if (!hs) return NSPB_ERR_ALLOC;
    cudaError_t e = cudaMemcpyAsync(&hs->c.err, d, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    *h = hs->c.err;
    return NSPB_OK;
  }
};

bool valid_in(const nspb_csr_in *M) {
  if (!M || M->nrows < 0 || M->ncols < 0 || M->nnz < 0 || M->nnz > INT32_MAX) return false;
  if (M->nrows > 0 && !M->rowptr) return false;
  if (M->nnz > 0 && (!M->col || !M->val)) return false;
  return M->val_type == NSPB_F64 || M->val_type == NSPB_F32;
}

}  // namespace
}  // namespace nspb

using namespace nspb;

extern "C" {

int nspb_transpose(const nspb_csr_in *A, nspb_csr_out *T, const nspb_opts *opts) {
  if (!valid_in(A) || !T) return NSPB_ERR_INVALID;
  if ((T->col || T->val) && (!T->col || !T->val)) return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NSPB_ERR_NO_DEVICE;
  }
  const size_t vsz = A->val_type == NSPB_F32 ? 4 : 8;
  const int64_t nnz = A->nnz;
  bool own_r = false, own_cv = false;
  int st = NSPB_OK;
  if (T->col && T->capacity < nnz) {
    T->nnz = nnz;
    return NSPB_ERR_CAPACITY;
  }
  if (!T->rowptr) {
    if ((st = alloc_out(reinterpret_cast<void **>(&T->rowptr), ((size_t)A->ncols + 1) * 4))) return st;
    own_r = true;
  }
  if (!T->col) {
    st = alloc_out(reinterpret_cast<void **>(&T->col), (size_t)nnz * 4);
    if (!st) {
      st = alloc_out(reinterpret_cast<void **>(&T->val), (size_t)nnz * vsz);
      if (st) {
        cudaFree(T->col);
        T->col = nullptr;
      }
    }
    if (!st) {
      own_cv = true;
      T->capacity = nnz;
    }
  }
  ErrWord ew;
  if (!st) {
    Scratch ws(s);
    st = ws.get(&ew.d, 1);
    if (!st) st = cuda_status(cudaMemsetAsync(ew.d, 0, sizeof(int), s));
    if (!st)
      st = vsz == 8 ? transpose_t<double>(A, T->rowptr, T->col, T->val, ew.d, s)
                    : transpose_t<float>(A, T->rowptr, T->col,
                                         reinterpret_cast<float *>(T->val), ew.d, s);
    int h = 0;
    if (!st) st = ew.read(s, &h);
    if (!st && h) st = NSPB_ERR_INVALID;  // a column outside [0, ncols)
  }
  if (st) {
    cudaStreamSynchronize(s);
    if (own_cv) {
      cudaFree(T->col);
      cudaFree(T->val);
      T->col = nullptr;
      T->val = nullptr;
    }
    if (own_r) {
      cudaFree(T->rowptr);
      T->rowptr = nullptr;
    }
    return st;
  }
  T->nrows = A->ncols;
  T->ncols = A->nrows;
  T->nnz = nnz;
  return NSPB_OK;
}

int nspb_sa_prolongator(const nspb_csr_in *A, const nspb_csr_in *Ptent, double omega,
                        nspb_csr_out *P, const nspb_opts *opts) {
  if (!valid_in(A) || !valid_in(Ptent) || !P) return NSPB_ERR_INVALID;
  if (A->val_type != NSPB_F64 || Ptent->val_type != NSPB_F64) return NSPB_ERR_INVALID;
  if (A->nrows != A->ncols || Ptent->nrows != A->nrows) return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  o.precision = NSPB_PREC_FP64;
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  const bool own_r = !P->rowptr, own_cv = !P->col;
  int st = nspb_spgemm(A, Ptent, P, &o, nullptr);  // P = A P_tent
  if (st) return st;
  const int n = A->nrows;
  auto smooth = [&]() -> int {
    Scratch ws(s);
    double *D = nullptr;
    ErrWord ew;
    int r;
    if ((r = ws.get(&D, (size_t)n)) || (r = ws.get(&ew.d, 1))) return r;
    if ((r = cuda_status(cudaMemsetAsync(ew.d, 0, sizeof(int), s)))) return r;
    k_diag<<<grid_for(n, 256), 256, 0, s>>>(A->rowptr, A->col,
                                            static_cast<const double *>(A->val), n, D, ew.d);
    if ((r = cuda_status(cudaGetLastError()))) return r;
    k_sa_smooth<<<grid_for((long long)n * 32, 256), 256, 0, s>>>(
        P->rowptr, P->col, P->val, Ptent->rowptr, Ptent->col,
        static_cast<const double *>(Ptent->val), D, omega, n, ew.d);
    if ((r = cuda_status(cudaGetLastError()))) return r;
    int h = 0;
    if ((r = ew.read(s, &h))) return r;
    return h ? NSPB_ERR_INVALID : NSPB_OK;  // a missing diagonal or tentative column
  };
  if (n > 0 && (st = smooth())) {
    cudaStreamSynchronize(s);
    if (own_cv) {
      cudaFree(P->col);
      cudaFree(P->val);
      P->col = nullptr;
      P->val = nullptr;
    }
    if (own_r) {
      cudaFree(P->rowptr);
      P->rowptr = nullptr;
    }
  }
  return st;
}

int nspb_galerkin(const nspb_csr_in *A, const nspb_csr_in *P, nspb_csr_out *R,
                  nspb_csr_out *Ac, const nspb_opts *opts) {
  if (!valid_in(A) || !valid_in(P) || !Ac) return NSPB_ERR_INVALID;
  if (A->ncols != P->nrows || A->nrows != P->nrows) return NSPB_ERR_INVALID;
  nspb_csr_out Rt = {};
  nspb_csr_out *r = R ? R : &Rt;
  int st = nspb_transpose(P, r, opts);
  if (st) return st;
  nspb_csr_out AP = {};
  st = nspb_spgemm(A, P, &AP, opts, nullptr);
  if (!st) {
    const nspb_csr_in rin = {r->nrows, r->ncols, r->nnz, r->rowptr, r->col, r->val,
                             P->val_type, 0};
    const nspb_csr_in apin = {AP.nrows, AP.ncols, AP.nnz, AP.rowptr, AP.col, AP.val,
                              NSPB_F64, 0};
    if (P->val_type == NSPB_F32) st = NSPB_ERR_UNSUPPORTED;  // R would be fp32, AP fp64
    else st = nspb_spgemm(&rin, &apin, Ac, opts, nullptr);
  }
  nspb_free(AP.rowptr);
  nspb_free(AP.col);
  nspb_free(AP.val);
  if (!R) {
    nspb_free(Rt.rowptr);
    nspb_free(Rt.col);
    nspb_free(Rt.val);
  }
  return st;
}

}  // extern "C"
