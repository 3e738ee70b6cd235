// Column remap for row-blocked products (getmct / compactcol / shrink).
//
// Reference counterparts (amavliut/nsp):
//   getmct          src/getmct.cu:41-92   thrust sort + unique of the columns
//                                          outside the local rows, list copied
//                                          to the host
//   compactcol      src/compactcol.cu:160-163 with src/cuCompactor.cuh:34-154
//                                          (block counts, thrust scan, scatter)
//   apply_mask_permut_GPU_noSideEffects   src/spspmpi.cu:58-84 (binary search)
// getmct here needs no sort: the selected columns set bits of a device
// bitmap, and the set bits are emitted in column order with the single-pass
// scan over per-word popcounts, which yields the sorted unique list directly.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "remap.h"
#include "spgemm_host.h"

namespace nspb {

constexpr int kCompactThreads = 256;
constexpr int kCompactItems = 16;
constexpr int kCompactTile = kCompactThreads * kCompactItems;

__device__ __forceinline__ bool outside(int c, int lo, int hi) { return c < lo || c > hi; }

__global__ void __launch_bounds__(kCompactThreads)
    k_tile_count(const int *__restrict__ in, long long n, int lo, int hi,
                 int *__restrict__ tile_counts) {
  const long long base = (long long)blockIdx.x * kCompactTile;
  int c = 0;
  for (int q = 0; q < kCompactItems; ++q) {
    const long long i = base + (long long)q * kCompactThreads + threadIdx.x;
    if (i < n) c += outside(in[i], lo, hi);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ int red[kCompactThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kCompactThreads / 32; ++w) s += red[w];
    tile_counts[blockIdx.x] = s;
  }
}

// Writes the selected items of each tile at its scanned offset, in order.
__global__ void __launch_bounds__(kCompactThreads)
    k_tile_scatter(const int *__restrict__ in, long long n, int lo, int hi,
                   const int *__restrict__ tile_off, int *__restrict__ out) {
  __shared__ int red[kCompactThreads / 32];
  const long long base = (long long)blockIdx.x * kCompactTile;
  int run = tile_off[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = 0; q < kCompactItems; ++q) {
    const long long i = base + (long long)q * kCompactThreads + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    const bool keep = i < n && outside(v, lo, hi);
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) red[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kCompactThreads / 32; ++w) {
      const int c = red[w];
      if (w < warp) before += c;
      total += c;
    }
    if (keep) out[run + before + __popc(m & ((1u << lane) - 1u))] = v;
    run += total;
    __syncthreads();
  }
}

// ---- getmct: bitmap of selected columns ---------------------------------------
__global__ void k_max_col(const int *__restrict__ col, long long n, int *__restrict__ mx) {
  int m = -1;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    m = max(m, col[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m >= 0) atomicMax(mx, m);
}

__global__ void k_set_bits(const int *__restrict__ col, long long n, int lo, int hi,
                           unsigned *__restrict__ bm) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = col[i];
    if (c >= 0 && outside(c, lo, hi)) {
      const unsigned bit = 1u << (c & 31);
      if (!(bm[c >> 5] & bit)) atomicOr(&bm[c >> 5], bit);
    }
  }
}

__global__ void k_word_pop(const unsigned *__restrict__ bm, int words, int *__restrict__ cnt) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < words) cnt[w] = __popc(bm[w]);
}

__global__ void k_emit_bits(const unsigned *__restrict__ bm, int words,
                            const int *__restrict__ off, int *__restrict__ out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  unsigned m = bm[w];
  int p = off[w];
  while (m) {
    const int b = __ffs(m) - 1;
    m &= m - 1u;
    out[p++] = w * 32 + b;
  }
}

// ---- shrink: position of each column in a sorted list ---------------------------
__global__ void k_shrink(const int *__restrict__ col, long long n, const int *__restrict__ cols,
                         long long ncols, int *__restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = col[i];
    long long lo = 0, hi = ncols;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (__ldg(cols + mid) < c) lo = mid + 1; else hi = mid;
    }
    out[i] = (lo < ncols && __ldg(cols + lo) == c) ? (int)lo : -1;
  }
}

static int grid_for(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  const long long cap = (long long)dev_info().sms * 32;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// Scratch for a compaction or a bitmap emission: counts + scanned offsets +
// a header (total, tile counter, error word, the scan's bin histogram) +
// scan tile states + an optional extra block.
struct RemapScratch {
  char *ws = nullptr;
  int *counts = nullptr, *offs = nullptr, *hdr_ctr = nullptr, *err = nullptr, *hist = nullptr;
  long long *total = nullptr;
  unsigned long long *tiles = nullptr;
  size_t bytes = 0;
};

static size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }

static int remap_scratch(RemapScratch &r, int items, size_t extra, cudaStream_t s) {
  const size_t o_counts = 0;
  const size_t o_offs = a256(o_counts + (size_t)(items + 1) * 4);
  const size_t o_hdr = a256(o_offs + (size_t)(items + 1) * 4);
  const size_t o_tiles = a256(o_hdr + 128);
  const size_t o_extra = a256(o_tiles + (size_t)scan_tiles(items) * 8);
  r.bytes = a256(o_extra + extra);
  int st = scratch_alloc(reinterpret_cast<void **>(&r.ws), r.bytes, s);
  if (st) return st;
  r.counts = reinterpret_cast<int *>(r.ws + o_counts);
  r.offs = reinterpret_cast<int *>(r.ws + o_offs);
  r.total = reinterpret_cast<long long *>(r.ws + o_hdr);
  r.hdr_ctr = reinterpret_cast<int *>(r.ws + o_hdr + 8);
  r.err = reinterpret_cast<int *>(r.ws + o_hdr + 12);
  r.hist = reinterpret_cast<int *>(r.ws + o_hdr + 16);
  r.tiles = reinterpret_cast<unsigned long long *>(r.ws + o_tiles);
  if (cudaMemsetAsync(r.ws + o_hdr, 0, o_extra - o_hdr, s) != cudaSuccess) {
    cudaGetLastError();
    return NSPB_ERR_CUDA;
  }
  return NSPB_OK;
}

static char *remap_extra(RemapScratch &r, int items) {
  const size_t o_offs = a256((size_t)(items + 1) * 4);
  const size_t o_hdr = a256(o_offs + (size_t)(items + 1) * 4);
  const size_t o_tiles = a256(o_hdr + 128);
  return r.ws + a256(o_tiles + (size_t)scan_tiles(items) * 8);
}

static int read_total(RemapScratch &r, int64_t *out, cudaStream_t s) {
  long long t = 0;
  int err = 0;
  if (cudaMemcpyAsync(&t, r.total, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&err, r.err, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    g_last_cuda = (int)cudaGetLastError();
    return NSPB_ERR_CUDA;
  }
  if (err) return NSPB_ERR_DEVICE;
  *out = t;
  return NSPB_OK;
}

int compactcol_dev(const int *d_in, int64_t n, int lo, int hi, int *d_out, int64_t *nout,
                   cudaStream_t s) {
  if (n == 0) {
    *nout = 0;
    return NSPB_OK;
  }
  const int tiles = (int)((n + kCompactTile - 1) / kCompactTile);
  RemapScratch r;
  int st = remap_scratch(r, tiles, 0, s);
  if (st) return st;
  k_tile_count<<<tiles, kCompactThreads, 0, s>>>(d_in, n, lo, hi, r.counts);
  cudaError_t e = launch_scan(r.counts, tiles, r.offs, r.total, r.tiles, r.hdr_ctr, bin_limits(0, 0),
                                  r.hist, r.err, s);
  if (e == cudaSuccess) {
    k_tile_scatter<<<tiles, kCompactThreads, 0, s>>>(d_in, n, lo, hi, r.offs, d_out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    scratch_free(r.ws, s);
    return NSPB_ERR_CUDA;
  }
  st = read_total(r, nout, s);
  scratch_free(r.ws, s);
  return st;
}

int getmct_dev(const int *d_col, int64_t nnz, int first, int last, int *d_out, int64_t *nout,
               cudaStream_t s) {
  if (nnz == 0) {
    *nout = 0;
    return NSPB_OK;
  }
  // largest column -> bitmap size
  int *d_mx = nullptr;
  int st = scratch_alloc(reinterpret_cast<void **>(&d_mx), 256, s);
  if (st) return st;
  int mx = -1;
  cudaMemsetAsync(d_mx, 0xff, 4, s);
  k_max_col<<<grid_for(nnz, 256), 256, 0, s>>>(d_col, nnz, d_mx);
  cudaMemcpyAsync(&mx, d_mx, 4, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  scratch_free(d_mx, s);
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    return NSPB_ERR_CUDA;
  }
  if (mx < 0) {
    *nout = 0;
    return NSPB_OK;
  }
  const int words = mx / 32 + 1;
  RemapScratch r;
  if ((st = remap_scratch(r, words, (size_t)words * 4, s))) return st;
  unsigned *bm = reinterpret_cast<unsigned *>(remap_extra(r, words));
  // outside(c, lo, hi) holds for every column when lo = INT_MAX, hi = -1
  const int lo = first > last ? 0x7fffffff : first;
  const int hi = first > last ? -1 : last;
  cudaMemsetAsync(bm, 0, (size_t)words * 4, s);
  k_set_bits<<<grid_for(nnz, 256), 256, 0, s>>>(d_col, nnz, lo, hi, bm);
  k_word_pop<<<(words + 255) / 256, 256, 0, s>>>(bm, words, r.counts);
  e = launch_scan(r.counts, words, r.offs, r.total, r.tiles, r.hdr_ctr, bin_limits(0, 0), r.hist,
                  r.err, s);
  if (e == cudaSuccess) {
    k_emit_bits<<<(words + 255) / 256, 256, 0, s>>>(bm, words, r.offs, d_out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    scratch_free(r.ws, s);
    return NSPB_ERR_CUDA;
  }
  st = read_total(r, nout, s);
  scratch_free(r.ws, s);
  return st;
}

int shrink_col_dev(const int *d_col, int64_t nnz, const int *d_cols, int64_t ncols, int *d_out,
                   cudaStream_t s) {
  if (nnz == 0) return NSPB_OK;
  k_shrink<<<grid_for(nnz, 256), 256, 0, s>>>(d_col, nnz, d_cols, ncols, d_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    return NSPB_ERR_CUDA;
  }
  return NSPB_OK;
}

}  // namespace nspb

using namespace nspb;

static bool have_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return false;
  }
  return true;
}

extern "C" int nspb_compactcol(const int32_t *d_in, int64_t n, int32_t lo, int32_t hi,
                               int32_t *d_out, int64_t *nout, void *stream) {
  if (n < 0 || !nout || (n > 0 && (!d_in || !d_out))) return NSPB_ERR_INVALID;
  if (!have_device()) return NSPB_ERR_NO_DEVICE;
  return compactcol_dev(d_in, n, lo, hi, d_out, nout, static_cast<cudaStream_t>(stream));
}

extern "C" int nspb_getmct(const int32_t *d_col, int64_t nnz, int32_t first, int32_t last,
                           int32_t *d_out, int64_t *nout, void *stream) {
  if (nnz < 0 || !nout || (nnz > 0 && (!d_col || !d_out))) return NSPB_ERR_INVALID;
  if (!have_device()) return NSPB_ERR_NO_DEVICE;
  return getmct_dev(d_col, nnz, first, last, d_out, nout, static_cast<cudaStream_t>(stream));
}

extern "C" int nspb_shrink_col(const int32_t *d_col, int64_t nnz, const int32_t *d_cols,
                               int64_t ncols, int32_t *d_out, void *stream) {
  if (nnz < 0 || ncols < 0 || (nnz > 0 && (!d_col || !d_out || (ncols > 0 && !d_cols))))
    return NSPB_ERR_INVALID;
  if (!have_device()) return NSPB_ERR_NO_DEVICE;
  return shrink_col_dev(d_col, nnz, d_cols, ncols, d_out, static_cast<cudaStream_t>(stream));
}
