// Row analysis kernels: B-row order check, intermediate-product counts and
// symbolic binning, bin permutation, and the single-pass row_ptr scan.
//
// Reference counterparts (amavliut/nsp):
//   nsp_set_intprod_num  nsp/src/nsp.cu:306-320   (one thread per row)
//   nsp_set_bin          nsp/src/nsp.cu:325-352   (10 global atomics per thread)
//   nsp_set_row_perm     nsp/src/nsp.cu:356-411   (one global atomic per row)
//   cub::DeviceScan::ExclusiveSum + D2H of nnz     nsp/src/nsp.cu:1124-1126
//   nsp_set_bin_min / nsp_set_row_perm_min          nsp/src/nsp.cu:1137-1237
// Here a row group of lanes reads each A row coalesced, bins are counted in
// shared memory with one global atomic per bin per block, and the scan is a
// single pass with decoupled look-back that also histograms the numeric bins.
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"

#include <algorithm>

namespace nspb {

// ---- bin limits ------------------------------------------------------------------
BinLimits bin_limits(int sym_fill_pct, int num_fill_pct) {
  const int sf = sym_fill_pct <= 0 ? 75 : std::min(std::max(sym_fill_pct, 10), 90);
  const int nf = num_fill_pct <= 0 ? 50 : std::min(std::max(num_fill_pct, 10), 50);
  BinLimits l;
  for (int b = 0; b < 16; ++b) {
    // bin b's table has 32 << b slots
    l.sym[b] = b < kSymLong ? std::max(1, (int)((32LL << b) * sf / 100)) : 0x7fffffff;
    l.num[b] = b < kNumLong ? std::max(1, (int)((32LL << b) * nf / 100)) : 0x7fffffff;
  }
  return l;
}
int sym_bin_of(int ub, const BinLimits &l) { return sym_bin(ub, l); }
int num_bin_of(int nz, const BinLimits &l) { return num_bin(nz, l); }

// ---- B row order --------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_check_sorted(const int *__restrict__ rpt, const int *__restrict__ col,
                   int n, int *__restrict__ flags) {
  const int row = (blockIdx.x * 256 + threadIdx.x) >> 3;
  const int lane = threadIdx.x & 7;
  int bad = 0;
  if (row < n) {
    const int s0 = rpt[row], s1 = rpt[row + 1];
    for (int e = s0 + lane; e + 1 < s1; e += 8) bad |= (col[e] >= col[e + 1]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags, B_UNSORTED);
}

cudaError_t launch_check_sorted(const CsrDev &B, int *flags, cudaStream_t s) {
  if (B.nrows <= 0) return cudaSuccess;
  const int grid = (int)(((int64_t)B.nrows * 8 + 255) / 256);
  k_check_sorted<<<grid, 256, 0, s>>>(B.rpt, B.col, B.nrows, flags);
  return cudaGetLastError();
}

// Every product's B: blockIdx.y is the product, blocks stride over its rows.
__global__ void __launch_bounds__(256)
    k_check_sorted_table(const Operands<void> *__restrict__ ops, int *__restrict__ flags) {
  const Operands<void> o = ops[blockIdx.y];
  int bad = 0;
  for (int r0 = blockIdx.x * 32; r0 < o.brows; r0 += gridDim.x * 32) {  // block-uniform
    const int row = r0 + (int)(threadIdx.x >> 3);
    const int lane = threadIdx.x & 7;
    if (row < o.brows) {
      const int s0 = o.brpt[row], s1 = o.brpt[row + 1];
      for (int e = s0 + lane; e + 1 < s1; e += 8) bad |= (o.bcol[e] >= o.bcol[e + 1]);
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags, B_UNSORTED);
}

cudaError_t launch_check_sorted_table(const Operands<void> *ops, int nprod, int max_brows,
                                      int *flags, cudaStream_t s) {
  if (nprod <= 0 || max_brows <= 0) return cudaSuccess;
  const int gx = (int)std::min<int64_t>(((int64_t)max_brows + 31) / 32, 1024);
  k_check_sorted_table<<<dim3(gx, nprod), 256, 0, s>>>(ops, flags);
  return cudaGetLastError();
}

// ---- intermediate products and symbolic bins ---------------------------------
// A rows longer than this are counted by a whole block (k_rowinfo_long), so
// a power-law row of 10^4 entries does not leave one lane group walking it.
constexpr int kRowinfoLong = 1024;

template <int GA, bool MULTI>
__global__ void __launch_bounds__(256)
    k_rowinfo(const ProdTable<void> src, int n, const BinLimits lim,
              int *__restrict__ row_nz, int64_t *__restrict__ row_ip,
              int *__restrict__ sym_counts,
              unsigned long long *__restrict__ total_ip, int *__restrict__ flags,
              int *__restrict__ long_list, int *__restrict__ long_count) {
  // With flags (B is A): the order of every row read here is checked too,
  // which is the B check of launch_check_sorted without a second read.
  // persistent grid: bin counts and the total accumulate in shared memory and
  // reach global memory once per block (one block per few rows made every
  // block add into the same dozen counters)
  __shared__ int hist[kSymBins];
  __shared__ unsigned long long s_total;
  if (threadIdx.x < kSymBins) hist[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_total = 0ull;
  __syncthreads();
  auto tile = cg::tiled_partition<GA>(cg::this_thread_block());
  const int lane = tile.thread_rank();
  constexpr int kGroups = 256 / GA;
  unsigned long long my_total = 0;
  int bad = 0;
  for (int row = blockIdx.x * kGroups + (int)threadIdx.x / GA; row < n;
       row += gridDim.x * kGroups) {
    Operands<void> o;
    const int lr = prod_row<MULTI>(src, row, o);
    const int a0 = o.arpt[lr], a1 = o.arpt[lr + 1];
    if (long_list && a1 - a0 > kRowinfoLong) {  // left to k_rowinfo_long
      if (lane == 0) long_list[atomicAdd(long_count, 1)] = row;
      continue;
    }
    long long ip = 0;
    for (int j = a0 + lane; j < a1; j += GA) {
      const int k = ld_stream(o.acol + j);
      ip += o.brpt[k + 1] - o.brpt[k];
      // each entry against its predecessor, read directly: no dependence
      // between rounds, so long rows keep their loads in flight
      if (flags && j > a0 && k <= __ldg(o.acol + j - 1)) bad = 1;
    }
    ip = cg::reduce(tile, ip, cg::plus<long long>());
    if (lane == 0) {
      const int ub = (int)(ip < (long long)o.ncols ? ip : (long long)o.ncols);
      row_nz[row] = ub;
      if (row_ip) row_ip[row] = ip;
      if (ub > 0) atomicAdd(&hist[sym_bin(ub, lim)], 1);
      my_total += (unsigned long long)ip;
    }
  }
  if (lane == 0 && my_total) atomicAdd(&s_total, my_total);
  if (__syncthreads_or(bad) && flags && threadIdx.x == 0) atomicOr(flags, B_UNSORTED);
  if (threadIdx.x < kSymBins && hist[threadIdx.x])
    atomicAdd(&sym_counts[threadIdx.x], hist[threadIdx.x]);
  if (threadIdx.x == 0 && s_total) atomicAdd(total_ip, s_total);
}

// The rows k_rowinfo listed: one block per row, the same outputs.
template <bool MULTI>
__global__ void __launch_bounds__(256)
    k_rowinfo_long(const ProdTable<void> src, const BinLimits lim, const int *__restrict__ long_list,
                   const int *__restrict__ long_count, int *__restrict__ row_nz,
                   int64_t *__restrict__ row_ip, int *__restrict__ sym_counts,
                   unsigned long long *__restrict__ total_ip, int *__restrict__ flags) {
  __shared__ int hist[kSymBins];
  __shared__ long long red[8];
  __shared__ unsigned long long s_total;
  if (threadIdx.x < kSymBins) hist[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_total = 0ull;
  __syncthreads();
  const int count = *long_count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int bad = 0;
  for (int q = blockIdx.x; q < count; q += gridDim.x) {  // uniform across the block
    const int row = long_list[q];
    Operands<void> o;
    const int lr = prod_row<MULTI>(src, row, o);
    const int a0 = o.arpt[lr], a1 = o.arpt[lr + 1];
    long long ip = 0;
    for (int j = a0 + (int)threadIdx.x; j < a1; j += 256) {
      const int k = ld_stream(o.acol + j);
      ip += o.brpt[k + 1] - o.brpt[k];
      if (flags && j > a0 && k <= __ldg(o.acol + j - 1)) bad = 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ip += __shfl_xor_sync(0xffffffffu, ip, o);
    if (lane == 0) red[warp] = ip;
    __syncthreads();
    if (threadIdx.x == 0) {
      long long t = 0;
      for (int w = 0; w < 8; ++w) t += red[w];
      const int ub = (int)(t < (long long)o.ncols ? t : (long long)o.ncols);
      row_nz[row] = ub;
      if (row_ip) row_ip[row] = t;
      if (ub > 0) atomicAdd(&hist[sym_bin(ub, lim)], 1);
      s_total += (unsigned long long)t;
    }
    __syncthreads();
  }
  if (__syncthreads_or(bad) && flags && threadIdx.x == 0) atomicOr(flags, B_UNSORTED);
  if (threadIdx.x < kSymBins && hist[threadIdx.x])
    atomicAdd(&sym_counts[threadIdx.x], hist[threadIdx.x]);
  if (threadIdx.x == 0 && s_total) atomicAdd(total_ip, s_total);
}

cudaError_t launch_rowinfo(const ProdTable<void> &t, int n, int64_t a_nnz, const BinLimits &lim,
                           int *row_nz,
                           int64_t *row_ip, int *sym_counts,
                           unsigned long long *total_ip, int *flags, int *long_list,
                           int *long_count, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const double avg = (double)a_nnz / (double)n;
  const int ga = avg > 24.0 ? 32 : avg > 12.0 ? 16 : avg > 6.0 ? 8 : 4;
  const int grid = (int)std::min<int64_t>(((int64_t)n * ga + 255) / 256,
                                          (int64_t)dev_info().sms * 8);
  const bool multi = t.prod_of_row != nullptr;
#define NSPB_RI(GA)                                                                         \
  (multi ? k_rowinfo<GA, true><<<grid, 256, 0, s>>>(t, n, lim, row_nz, row_ip, sym_counts, total_ip, \
                                                    flags, long_list, long_count)           \
         : k_rowinfo<GA, false><<<grid, 256, 0, s>>>(t, n, lim, row_nz, row_ip, sym_counts,       \
                                                     total_ip, flags, long_list, long_count))
  switch (ga) {
    case 32: NSPB_RI(32); break;
    case 16: NSPB_RI(16); break;
    case 8: NSPB_RI(8); break;
    default: NSPB_RI(4); break;
  }
#undef NSPB_RI
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !long_list) return e;
  auto klong = multi ? k_rowinfo_long<true> : k_rowinfo_long<false>;
  klong<<<dev_info().sms * 4, 256, 0, s>>>(t, lim, long_list, long_count, row_nz, row_ip, sym_counts,
                                           total_ip, flags);
  return cudaGetLastError();
}

// ---- bin permutation ------------------------------------------------------------
// Each block of 1024 rows lists its rows of every bin in ascending row order
// (a stable split: ranks inside a warp from __match_any_sync peers, warp
// offsets from a scan of the per-warp counts), at a place in the bin that one
// atomic per (block, bin) reserves. Runs of consecutive list entries are then
// runs of neighbouring rows, which the row templates of the entry-map kernels
// rely on (rows of a structured grid repeat their neighbours' pattern).
__global__ void __launch_bounds__(1024)
    k_perm(const int *__restrict__ key, int n, int kind, BinOffsets off, const BinLimits lim,
           int *__restrict__ cursor, int *__restrict__ perm) {
  __shared__ int wcnt[16][33];  // [bin][warp]: rows, then the warp's offset in the block
  __shared__ int base[16];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = threadIdx.x; t < 16 * 33; t += blockDim.x) (&wcnt[0][0])[t] = 0;
  const int i = blockIdx.x * 1024 + threadIdx.x;
  int b = -1;
  if (i < n) {
    const int k = kind == 0 ? key[i] : key[i + 1] - key[i];
    if (k > 0) b = kind == 0 ? sym_bin(k, lim) : num_bin(k, lim);
  }
  __syncthreads();
  const unsigned peers = __match_any_sync(0xffffffffu, b);
  const int rank = __popc(peers & ((1u << lane) - 1u));
  if (b >= 0 && rank == 0) wcnt[b][w] = __popc(peers);
  __syncthreads();
  if (w < 16) {  // warp w scans bin w over the block's 32 warps
    const int v = wcnt[w][lane];
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    wcnt[w][lane] = incl - v;
    if (lane == 31 && incl > 0) base[w] = off.v[w] + atomicAdd(&cursor[w], incl);
  }
  __syncthreads();
  if (b >= 0) perm[base[b] + wcnt[b][w] + rank] = i;
}

cudaError_t launch_perm(const int *key, int n, int kind, BinOffsets offsets, const BinLimits &lim,
                        int *cursor, int *perm, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_perm<<<(n + 1023) / 1024, 1024, 0, s>>>(key, n, kind, offsets, lim, cursor, perm);
  return cudaGetLastError();
}

// ---- heaviest rows first in the block-per-row bins ----------------------------
// A block-per-row kernel draws its rows from a ticket counter in list order,
// and k_perm lists a bin's rows in about row order. In a power-law matrix the
// hub rows then sit anywhere in the list: one drawn near the end keeps a
// single SM busy long after the others ran dry (a list-scheduling makespan of
// about 1.6x the ideal on the 1M-row power-law product). Reordering each list
// by descending weight class, floor(log2(weight)), gives the
// longest-processing-time-first schedule within a factor 2 per class. Rows of
// one class keep no particular order: each row is computed by one block on its
// own, so the order changes only which block takes it, never its result.
// One block per list, staged in shared memory; a list of more than
// kOrderCap rows is left as it is.
constexpr int kOrderThreads = 1024;

__global__ void __launch_bounds__(kOrderThreads)
    k_order_rows(const int *__restrict__ key, int kind, RowLists lists, int *__restrict__ perm) {
  extern __shared__ int s_rows[];
  __shared__ int cls[32];
  const int count = lists.count[blockIdx.x];
  if (count > kOrderCap) return;  // block-uniform
  int *rows = perm + lists.off[blockIdx.x];
  if (threadIdx.x < 32) cls[threadIdx.x] = 0;
  __syncthreads();
  auto weight_class = [&](int r) {
    const int w = kind == 0 ? key[r] : key[r + 1] - key[r];
    return 31 - __clz(max(w, 1));
  };
  for (int i = threadIdx.x; i < count; i += kOrderThreads) {
    const int r = rows[i];
    s_rows[i] = r;
    atomicAdd(&cls[weight_class(r)], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // heaviest class first
    int run = 0;
    for (int c = 31; c >= 0; --c) {
      const int k = cls[c];
      cls[c] = run;
      run += k;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < count; i += kOrderThreads) {
    const int r = s_rows[i];
    rows[atomicAdd(&cls[weight_class(r)], 1)] = r;
  }
}

cudaError_t launch_order_rows(const int *key, int kind, const RowLists &lists, int *perm,
                              cudaStream_t s) {
  int most = 0;
  for (int i = 0; i < lists.n; ++i) most = std::max(most, std::min(lists.count[i], kOrderCap));
  if (lists.n <= 0 || most <= 1) return cudaSuccess;
  const int smem = most * (int)sizeof(int);
  if (smem > 48 * 1024 && !allow_smem((const void *)k_order_rows)) return cudaErrorInvalidValue;
  k_order_rows<<<lists.n, kOrderThreads, smem, s>>>(key, kind, lists, perm);
  return cudaGetLastError();
}

// ---- single-pass exclusive scan with decoupled look-back -----------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr unsigned long long kAggregate = 1ull, kInclusive = 2ull;
constexpr int kWaitLimit = 1 << 22;  // ~0.3 s of polling before the error word is set

int scan_tiles(int n) { return n <= 0 ? 1 : (n + kScanTile - 1) / kScanTile; }

__device__ __forceinline__ void publish(unsigned long long *st, int t, long long v,
                                        unsigned long long flag) {
  *((volatile unsigned long long *)(st + t)) = ((unsigned long long)v << 2) | flag;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan(const int *__restrict__ in, int n, int *__restrict__ out,
           long long *__restrict__ total, unsigned long long *tile_state,
           int *tile_ctr, const BinLimits lim, int *__restrict__ num_counts,
           int *__restrict__ err) {
  __shared__ int s_tile;
  __shared__ long long s_warp[kScanThreads / 32];
  __shared__ long long s_prefix;
  __shared__ int hist[kNumBins];
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1);
  if (threadIdx.x < kNumBins) hist[threadIdx.x] = 0;
  __syncthreads();
  const int tile = s_tile;
  const long long base = (long long)tile * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  if (base + kScanItems <= n) {
    const int4 *p = reinterpret_cast<const int4 *>(in + base);
    const int4 x = p[0], y = p[1];
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
  } else {
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) v[q] = base + q < n ? in[base + q] : 0;
  }
  long long sum = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    sum += v[q];
    if (v[q] > 0) atomicAdd(&hist[num_bin(v[q], lim)], 1);
  }
  // block scan of the per-thread sums
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < kScanThreads / 32) s_warp[lane] = w;  // inclusive warp prefixes
  }
  __syncthreads();
  const long long block_total = s_warp[kScanThreads / 32 - 1];
  const long long excl = (warp ? s_warp[warp - 1] : 0) + incl - sum;
  if (threadIdx.x == 0) {
    long long prefix = 0;
    if (tile == 0) {
      publish(tile_state, 0, block_total, kInclusive);
    } else {
      publish(tile_state, tile, block_total, kAggregate);
      for (int p = tile - 1; p >= 0; --p) {
        unsigned long long st = *((volatile unsigned long long *)(tile_state + p));
        int spins = 0;
        while ((st & 3ull) == 0ull) {
          if (++spins > kWaitLimit) {
            atomicOr(err, ERR_WAIT);
            st = kInclusive;  // give up: treat as a zero inclusive prefix
            break;
          }
          __nanosleep(64);
          st = *((volatile unsigned long long *)(tile_state + p));
        }
        prefix += (long long)(st >> 2);
        if ((st & 3ull) == kInclusive) break;
      }
      publish(tile_state, tile, prefix + block_total, kInclusive);
    }
    s_prefix = prefix;
  }
  __syncthreads();
  long long run = s_prefix + excl;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    if (base + q < n) out[base + q] = run > 0x7fffffffLL ? 0x7fffffff : (int)run;
    run += v[q];
  }
  if (base < n && base + kScanItems >= n) {  // the thread holding row n-1
    out[n] = run > 0x7fffffffLL ? 0x7fffffff : (int)run;
    *total = run;
  }
  __syncthreads();
  if (threadIdx.x < kNumBins && hist[threadIdx.x])
    atomicAdd(&num_counts[threadIdx.x], hist[threadIdx.x]);
}

cudaError_t launch_scan(const int *row_nz, int n, int *crpt, long long *total,
                        unsigned long long *tile_state, int *tile_ctr, const BinLimits &lim,
                        int *num_counts, int *err, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_scan<<<scan_tiles(n), kScanThreads, 0, s>>>(row_nz, n, crpt, total, tile_state,
                                                tile_ctr, lim, num_counts, err);
  return cudaGetLastError();
}

// ---- numeric bins from an existing row pointer ---------------------------------
__global__ void __launch_bounds__(1024)
    k_num_hist(const int *__restrict__ crpt, int n, const BinLimits lim,
               int *__restrict__ num_counts) {
  __shared__ int hist[kNumBins];
  if (threadIdx.x < kNumBins) hist[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * 1024 + threadIdx.x;
  if (i < n) {
    const int k = crpt[i + 1] - crpt[i];
    if (k > 0) atomicAdd(&hist[num_bin(k, lim)], 1);
  }
  __syncthreads();
  if (threadIdx.x < kNumBins && hist[threadIdx.x])
    atomicAdd(&num_counts[threadIdx.x], hist[threadIdx.x]);
}

cudaError_t launch_num_hist(const int *crpt, int n, const BinLimits &lim, int *num_counts,
                            cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_num_hist<<<(n + 1023) / 1024, 1024, 0, s>>>(crpt, n, lim, num_counts);
  return cudaGetLastError();
}

}  // namespace nspb
