// Numeric phase: values of C, columns ascending within each row.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu):
//   nsp_calculate_value_col_bin_mpwarp     :1307-1401 (4/8/16 threads per row)
//   nsp_calculate_value_col_bin_each_warp  :1405-1494
//   nsp_calculate_value_col_bin_each_tb    :1499-1627 (block per row)
//   ..._each_tb_outsort + nsp_calc_val_sort_rows  :1632-1714,
//                                          nsp_calc_val_sort_rows.cu:24-527
//   ..._chunk_dynamic / nsp_calc_C_dense / ..._chunk_B_dense :1725-2151
// The reference sorts each row by an O(nnz^2) rank count. Here each row is
// sorted by a monotone bucket scatter over [min col, max col] followed by a
// rank count inside each bucket, in shared memory, and written coalesced.
//
// Row groups of G lanes walk the A row in order and cover one B row per step
// (B rows hold no repeated column when `owned`), so each slot of the hash
// table has a single writer per step: values are accumulated with plain
// read-modify-writes in A-row order, which makes the sums deterministic and
// equal, bit for bit, to a sequential Gustavson product that adds the rounded
// products a_ik*b_kj in the same order.
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"
#include "spgemm_host.h"

#include <algorithm>

namespace nspb {

// Device memory the long-row kernel may use for its per-CTA accumulators.
constexpr long long kDenseBudget = 4LL << 30;

// Rank of `key` among the bucket-ordered keys bk[0..n): its bucket spans
// [st, en). Reads 4 keys per shared-memory load from st rounded down to a
// multiple of 4: keys before st lie in earlier buckets, so they are smaller
// and are counted (the base is u0, not st); keys from en on lie in later
// buckets and are larger, so they are not; indices >= n are masked out.
// bk must be 16-byte aligned.
__device__ __forceinline__ int rank_in_bucket(const int *bk, int st, int en, int n, int key) {
  const int u0 = st & ~3;
  int rank = u0;
  for (int u = u0; u < en; u += 4) {
    const int4 v = *reinterpret_cast<const int4 *>(bk + u);
    rank += (v.x < key) + ((u + 1 < n) & (v.y < key)) + ((u + 2 < n) & (v.z < key)) +
            ((u + 3 < n) & (v.w < key));
  }
  return rank;
}

// ---- row groups -------------------------------------------------------------------
template <int G, int LOG2T>
struct NumGroupCfg {
  static constexpr int T = 1 << LOG2T;  // hash slots
  static constexpr int H = T / 2;       // max entries of a row in this bin
  static constexpr int NB = T / 2;      // sort buckets
  // per-group stride, rounded to 16 bytes so every group's fp64 arrays stay
  // 8-byte aligned
  // the table's upper half doubles as the bucket buffer of the sort
  static constexpr int BYTES = (T * 12 + NB * 4 + 15) & ~15;
  static constexpr int kBySmem = (56 * 1024) / BYTES > 0 ? (56 * 1024) / BYTES : 1;
  static constexpr int GPC = kBySmem < 256 / G ? kBySmem : 256 / G;
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * BYTES;
  static constexpr int PER = NB >= G ? NB / G : 1;  // scan counters per lane
};

// Compensated-mode parameters of a numeric launch (fp32 inputs).
struct CompArgs {
  int nmax;        // rows with at most nmax A entries accumulate error-free in
                   // fp32 pairs; longer rows accumulate in fp64
  int *redo;       // counter of rows accumulated in fp64
  int *max_deg;    // largest A-row degree among the pair-accumulated rows
};

// VT: value type of A and B (double, or float in the compensated mode).
// COMP: fp32 inputs with the error-free pair accumulation for short rows.
template <int G, int LOG2T, bool OWNED, typename VT, bool COMP>
__global__ void __launch_bounds__(256)
    k_num_group(const int *__restrict__ arpt, const int *__restrict__ acol,
                const VT *__restrict__ aval, const int *__restrict__ brpt,
                const int *__restrict__ bcol, const VT *__restrict__ bval,
                const int *__restrict__ crpt, int *__restrict__ ccol,
                double *__restrict__ cval, const int *__restrict__ rows, int count,
                int *__restrict__ err, CompArgs comp) {
  using C = NumGroupCfg<G, LOG2T>;
  extern __shared__ __align__(16) unsigned char smem_num[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  unsigned char *gb = smem_num + (size_t)g * C::BYTES;
  double *vals = reinterpret_cast<double *>(gb);
  int *keys = reinterpret_cast<int *>(vals + C::T);
  int *cnt = keys + C::T;

  int my_max_deg = 0, my_redo = 0;  // compensated mode, flushed once per group
  for (int r = blockIdx.x * C::GPC + g; r < count; r += gridDim.x * C::GPC) {
    const int row = rows ? rows[r] : r;
#pragma unroll 4
    for (int s = lane; s < C::T; s += G) {
      keys[s] = kEmpty;
      vals[s] = 0.0;
    }
    tile.sync();
    const int a0 = arpt[row], a1 = arpt[row + 1];
    // compensated mode: pair accumulation when the row's Dot2 bound allows it
    const bool pair = COMP && OWNED && (a1 - a0) <= comp.nmax;
    float2 *vals2 = reinterpret_cast<float2 *>(vals);
    int mn = 0x7fffffff, mx = -1;
    for (int ab = a0; ab < a1; ab += G) {
      int bs = 0, be = 0;
      double av = 0.0;
      if (ab + lane < a1) {
        const int k = ld_stream(acol + ab + lane);
        av = ldv_stream(aval + ab + lane);
        bs = __ldg(brpt + k);
        be = __ldg(brpt + k + 1);
      }
      const int na = min(G, a1 - ab);
      for (int t = 0; t < na; ++t) {
        const int s0 = tile.shfl(bs, t), s1 = tile.shfl(be, t);
        const double a = tile.shfl(av, t);
        for (int base = s0; base < s1; base += G) {
          const int e = base + lane;
          if (e < s1) {
            const int key = __ldg(bcol + e);
            if (pair) {
              const int h = num_slot<LOG2T>(keys, key, err);
              if (h >= 0) {
                float2 sc = vals2[h];
                comp_add(sc, (float)a, __ldg(reinterpret_cast<const float *>(bval) + e));
                vals2[h] = sc;
              }
            } else {
              num_insert<LOG2T, OWNED>(keys, vals, key, __dmul_rn(a, ldv(bval + e)), err);
            }
            mn = min(mn, key);
            mx = max(mx, key);
          }
          if (OWNED) tile.sync();  // next step may hit the same slot
        }
      }
    }
    tile.sync();
    if (COMP) {
      if (pair) {  // collapse each (s, c) pair to fp64
        for (int s = lane; s < C::T; s += G) {
          if (keys[s] >= 0) {
            const float2 sc = vals2[s];
            vals[s] = (double)sc.x + (double)sc.y;
          }
        }
        my_max_deg = max(my_max_deg, a1 - a0);
      } else {
        ++my_redo;
      }
      tile.sync();
    }
    const int c0 = crpt[row];
    const int n = crpt[row + 1] - c0;
    mn = cg::reduce(tile, mn, cg::less<int>());
    mx = cg::reduce(tile, mx, cg::greater<int>());
    // -- bucket sort. (1) compact the occupied slots to the front of the
    // table in slot order while counting buckets; (2) scan the counts;
    // (3) scatter into the table's free upper half [H, H+n); (4) rank inside
    // each bucket, writing the sorted row back to [0, n).
    for (int b = lane; b < C::NB; b += G) cnt[b] = 0;
    tile.sync();
    const float scale = n > 0 ? (float)C::NB / (float)((long long)mx - mn + 1) : 0.f;
    int occ_total = 0;
    for (int base = 0; base < C::T; base += G) {
      const int key = keys[base + lane];
      const double v = vals[base + lane];
      const unsigned ball = tile.ballot(key >= 0);
      tile.sync();  // every lane has read its slot before any slot is rewritten
      if (key >= 0) {
        const int pos = occ_total + __popc(ball & ((1u << lane) - 1u));
        keys[pos] = key;
        vals[pos] = v;
        atomicAdd(&cnt[bucket_of(key, mn, scale, C::NB)], 1);
      }
      occ_total += __popc(ball);
      tile.sync();
    }
    if constexpr (C::PER <= 8) {  // each lane scans a run of PER counters in registers
      int local[C::PER];
      int sum = 0;
#pragma unroll
      for (int q = 0; q < C::PER; ++q) {
        const int idx = lane * C::PER + q;
        local[q] = idx < C::NB ? cnt[idx] : 0;
        sum += local[q];
      }
      int ex = cg::exclusive_scan(tile, sum, cg::plus<int>());
#pragma unroll
      for (int q = 0; q < C::PER; ++q) {
        const int idx = lane * C::PER + q;
        if (idx < C::NB) cnt[idx] = ex;
        ex += local[q];
      }
    } else {  // rounds of G consecutive counters
      int run = 0;
      for (int base = 0; base < C::NB; base += G) {
        const int v = cnt[base + lane];
        const int incl = cg::inclusive_scan(tile, v, cg::plus<int>());
        cnt[base + lane] = run + incl - v;
        run += tile.shfl(incl, G - 1);
      }
    }
    tile.sync();
    if (occ_total != n || n > C::H) {  // symbolic/numeric disagreement: skip the row
      if (lane == 0) atomicOr(err, ERR_COUNT);
      tile.sync();
      continue;
    }
    int *bkeys = keys + C::H;
    double *bvals = vals + C::H;
    for (int q = lane; q < n; q += G) {
      const int key = keys[q];
      const int pos = atomicAdd(&cnt[bucket_of(key, mn, scale, C::NB)], 1);
      bkeys[pos] = key;
      bvals[pos] = vals[q];
    }
    tile.sync();
    for (int q = lane; q < n; q += G) {
      const int key = bkeys[q];
      const int b = bucket_of(key, mn, scale, C::NB);
      const int st = b ? cnt[b - 1] : 0, en = cnt[b];
      const int rank = rank_in_bucket(bkeys, st, en, n, key);
      keys[rank] = key;
      vals[rank] = bvals[q];
    }
    tile.sync();
    for (int q = lane; q < n; q += G) {
      ccol[c0 + q] = keys[q];
      cval[c0 + q] = vals[q];
    }
    tile.sync();
  }
  if (COMP && lane == 0) {
    if (my_max_deg) atomicMax(comp.max_deg, my_max_deg);
    if (my_redo) atomicAdd(comp.redo, my_redo);
  }
}

// ---- block per row: warps over A entries, atomic accumulation ----------------------
constexpr int kNumBlockThreads = 512;

// Exclusive scan of one int per thread over a 512-thread block; returns the
// thread's exclusive prefix and the block total in *tot. red: 16 ints.
__device__ __forceinline__ int block_exclusive_scan(int v, int *red, int *tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) red[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? red[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < (int)(blockDim.x >> 5)) red[lane] = w;
  }
  __syncthreads();
  *tot = red[(blockDim.x >> 5) - 1];
  const int r = (warp ? red[warp - 1] : 0) + incl - v;
  __syncthreads();
  return r;
}

template <int LOG2T, typename VT>
__global__ void __launch_bounds__(kNumBlockThreads)
    k_num_block(const int *__restrict__ arpt, const int *__restrict__ acol,
                const VT *__restrict__ aval, const int *__restrict__ brpt,
                const int *__restrict__ bcol, const VT *__restrict__ bval,
                const int *__restrict__ crpt, int *__restrict__ ccol,
                double *__restrict__ cval, const int *__restrict__ rows, int count,
                int *__restrict__ err, int *__restrict__ redo) {
  constexpr int T = 1 << LOG2T, H = T / 2, NB = T / 2;
  constexpr int PER = NB / kNumBlockThreads;
  extern __shared__ __align__(16) unsigned char smem_num[];
  double *vals = reinterpret_cast<double *>(smem_num);
  double *bvals = vals + T;
  int *keys = reinterpret_cast<int *>(bvals + H);
  int *bkeys = keys + T;
  int *cnt = bkeys + H;
  __shared__ int red[kNumBlockThreads / 32];
  __shared__ int s_mn, s_mx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kNumBlockThreads / 32;
  int rows_done = 0;
  for (int r = blockIdx.x; r < count; r += gridDim.x) {
    const int row = rows ? rows[r] : r;
    for (int s = threadIdx.x; s < T; s += kNumBlockThreads) {
      keys[s] = kEmpty;
      vals[s] = 0.0;
    }
    for (int b = threadIdx.x; b < NB; b += kNumBlockThreads) cnt[b] = 0;
    if (threadIdx.x == 0) {
      s_mn = 0x7fffffff;
      s_mx = -1;
    }
    __syncthreads();
    const int a0 = arpt[row], a1 = arpt[row + 1];
    int mn = 0x7fffffff, mx = -1;
    for (int j = a0 + warp; j < a1; j += W) {
      const int k = ld_stream(acol + j);
      const double a = ldv_stream(aval + j);
      const int s0 = __ldg(brpt + k), s1 = __ldg(brpt + k + 1);
      for (int e = s0 + lane; e < s1; e += 32) {
        const int key = __ldg(bcol + e);
        num_insert<LOG2T, false>(keys, vals, key, __dmul_rn(a, ldv(bval + e)), err);
        mn = min(mn, key);
        mx = max(mx, key);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
      atomicMin(&s_mn, mn);
      atomicMax(&s_mx, mx);
    }
    ++rows_done;  // compensated mode: every row here is an fp64 row
    __syncthreads();
    mn = s_mn;
    mx = s_mx;
    const int c0 = crpt[row];
    const int n = crpt[row + 1] - c0;
    const float scale = n > 0 ? (float)NB / (float)((long long)mx - mn + 1) : 0.f;
    for (int s = threadIdx.x; s < T; s += kNumBlockThreads) {
      const int key = keys[s];
      if (key >= 0) atomicAdd(&cnt[bucket_of(key, mn, scale, NB)], 1);
    }
    __syncthreads();
    int local[PER];
    int sum = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      local[q] = cnt[threadIdx.x * PER + q];
      sum += local[q];
    }
    int tot;
    int ex = block_exclusive_scan(sum, red, &tot);
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      cnt[threadIdx.x * PER + q] = ex;
      ex += local[q];
    }
    __syncthreads();
    if (tot != n || n > H) {
      if (threadIdx.x == 0) atomicOr(err, ERR_COUNT);
      __syncthreads();
      continue;
    }
    for (int s = threadIdx.x; s < T; s += kNumBlockThreads) {
      const int key = keys[s];
      if (key >= 0) {
        const int pos = atomicAdd(&cnt[bucket_of(key, mn, scale, NB)], 1);
        bkeys[pos] = key;
        bvals[pos] = vals[s];
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += kNumBlockThreads) {
      const int key = bkeys[q];
      const int b = bucket_of(key, mn, scale, NB);
      const int st = b ? cnt[b - 1] : 0, en = cnt[b];
      const int rank = rank_in_bucket(bkeys, st, en, n, key);
      keys[rank] = key;
      vals[rank] = bvals[q];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += kNumBlockThreads) {
      ccol[c0 + q] = keys[q];
      cval[c0 + q] = vals[q];
    }
    __syncthreads();
  }
  if (redo && threadIdx.x == 0 && rows_done) atomicAdd(redo, rows_done);
}

// ---- longest rows: dense column windows in shared memory ----------------------------
constexpr int kNumLongThreads = 1024;
constexpr int kWin = 16384;            // columns per window: 128 KB of fp64
constexpr int kWinWords = kWin / 32;   // occupancy bitmap

__device__ __forceinline__ int lower_bound_col(const int *__restrict__ col, int lo, int hi, int c) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(col + mid) < c) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <typename VT>
__global__ void __launch_bounds__(kNumLongThreads)
    k_num_long(const int *__restrict__ arpt, const int *__restrict__ acol,
               const VT *__restrict__ aval, const int *__restrict__ brpt,
               const int *__restrict__ bcol, const VT *__restrict__ bval,
               int ncols, bool sorted, const int *__restrict__ crpt,
               int *__restrict__ ccol, double *__restrict__ cval,
               const int *__restrict__ rows, int count, int *__restrict__ err,
               int *__restrict__ redo) {
  extern __shared__ __align__(16) unsigned char smem_num[];
  double *dense = reinterpret_cast<double *>(smem_num);
  unsigned *bm = reinterpret_cast<unsigned *>(dense + kWin);
  __shared__ int red[kNumLongThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kNumLongThreads / 32;
  int rows_done = 0;
  for (int r = blockIdx.x; r < count; r += gridDim.x) {
    const int row = rows ? rows[r] : r;
    const int a0 = arpt[row], a1 = arpt[row + 1];
    const bool per_thread = (a1 - a0) >= kNumLongThreads;
    int off = crpt[row];
    const int row_end = crpt[row + 1];
    for (int w0 = 0; w0 < ncols; w0 += kWin) {
      const int w1 = w0 + kWin;
      for (int s = threadIdx.x; s < kWin; s += kNumLongThreads) dense[s] = 0.0;
      for (int s = threadIdx.x; s < kWinWords; s += kNumLongThreads) bm[s] = 0u;
      __syncthreads();
      if (per_thread) {  // one A entry per thread
        for (int j = a0 + threadIdx.x; j < a1; j += kNumLongThreads) {
          const int k = ld_stream(acol + j);
          const double a = ldv_stream(aval + j);
          const int s1 = __ldg(brpt + k + 1);
          int e = __ldg(brpt + k);
          if (sorted) e = lower_bound_col(bcol, e, s1, w0);
          for (; e < s1; ++e) {
            const int c = __ldg(bcol + e);
            if (sorted && c >= w1) break;
            const unsigned d = (unsigned)(c - w0);
            if (d < (unsigned)kWin) {
              atomicAdd(dense + d, __dmul_rn(a, ldv(bval + e)));
              const unsigned bit = 1u << (d & 31u);
              if (!(bm[d >> 5] & bit)) atomicOr(bm + (d >> 5), bit);
            }
          }
        }
      } else {  // one A entry per warp, lanes over the B row
        for (int j = a0 + warp; j < a1; j += W) {
          const int k = ld_stream(acol + j);
          const double a = ldv_stream(aval + j);
          const int s1 = __ldg(brpt + k + 1);
          int e0 = __ldg(brpt + k);
          if (sorted) e0 = lower_bound_col(bcol, e0, s1, w0);
          for (int e = e0 + lane; e < s1; e += 32) {
            const int c = __ldg(bcol + e);
            if (sorted && c >= w1) break;
            const unsigned d = (unsigned)(c - w0);
            if (d < (unsigned)kWin) {
              atomicAdd(dense + d, __dmul_rn(a, ldv(bval + e)));
              const unsigned bit = 1u << (d & 31u);
              if (!(bm[d >> 5] & bit)) atomicOr(bm + (d >> 5), bit);
            }
          }
        }
      }
      __syncthreads();
      // compaction in column order: thread t owns bitmap word t
      const unsigned word = threadIdx.x < kWinWords ? bm[threadIdx.x] : 0u;
      const int pc = __popc(word);
      int incl = pc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) red[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        int v = red[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += t;
        }
        red[lane] = v;
      }
      __syncthreads();
      const int wtot = red[W - 1];
      int pos = off + (warp ? red[warp - 1] : 0) + incl - pc;
      unsigned m = word;
      if (pos + pc > row_end) {  // more entries than the symbolic count: write nothing
        if (pc) atomicOr(err, ERR_COUNT);
        m = 0u;
      }
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1u;
        const int d = threadIdx.x * 32 + b;
        ccol[pos] = w0 + d;
        cval[pos] = dense[d];
        ++pos;
      }
      off += wtot;
      __syncthreads();
    }
    if (threadIdx.x == 0 && off != row_end) atomicOr(err, ERR_COUNT);
    ++rows_done;  // compensated mode: every row here is an fp64 row
  }
  if (redo && threadIdx.x == 0 && rows_done) atomicAdd(redo, rows_done);
}

// ---- longest rows: dense fp64 accumulator in global memory ---------------------
// Each CTA owns an ncols-long fp64 accumulator in device memory (zero between
// rows) and a shared-memory bitmap over a 2^20-column window. Products are
// added with global fp64 atomics (one pass over the row's products for
// ncols <= 2^20), then the set bits are emitted in column order, each value
// read and its slot zeroed. acc is read and written with .cg accesses (L2
// only) so no stale L1 line is seen after another thread's atomic.
constexpr int kDenseBits = 1 << 20;
constexpr int kDenseWords = kDenseBits / 32;

template <typename VT>
__global__ void __launch_bounds__(kNumLongThreads)
    k_num_long_dense(const int *__restrict__ arpt, const int *__restrict__ acol,
                     const VT *__restrict__ aval, const int *__restrict__ brpt,
                     const int *__restrict__ bcol, const VT *__restrict__ bval, int ncols,
                     const int *__restrict__ crpt, int *__restrict__ ccol,
                     double *__restrict__ cval, const int *__restrict__ rows, int count,
                     double *__restrict__ acc_all, int *__restrict__ err,
                     int *__restrict__ redo) {
  extern __shared__ __align__(16) unsigned bm_dense[];
  __shared__ int red[kNumLongThreads / 32];
  double *acc = acc_all + (size_t)blockIdx.x * (size_t)ncols;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kNumLongThreads / 32;
  int rows_done = 0;
  for (int r = blockIdx.x; r < count; r += gridDim.x) {
    const int row = rows ? rows[r] : r;
    const int a0 = arpt[row], a1 = arpt[row + 1];
    int off = crpt[row];
    const int row_end = crpt[row + 1];
    for (int w0 = 0; w0 < ncols; w0 += kDenseBits) {
      const int wn = min(kDenseBits, ncols - w0);
      const int words = (wn + 31) >> 5;
      for (int q = threadIdx.x; q < words; q += kNumLongThreads) bm_dense[q] = 0u;
      __syncthreads();
      for (int j = a0 + warp; j < a1; j += W) {
        const int k = ld_stream(acol + j);
        const double a = ldv_stream(aval + j);
        const int s0 = __ldg(brpt + k), s1 = __ldg(brpt + k + 1);
        for (int e = s0 + lane; e < s1; e += 32) {
          const int c = __ldg(bcol + e);
          const unsigned d = (unsigned)(c - w0);
          if (d < (unsigned)wn) {
            atomicAdd(acc + c, __dmul_rn(a, ldv(bval + e)));
            const unsigned bit = 1u << (d & 31u);
            if (!(bm_dense[d >> 5] & bit)) atomicOr(bm_dense + (d >> 5), bit);
          }
        }
      }
      __threadfence_block();
      __syncthreads();
      // emit in column order, one round of kNumLongThreads words at a time
      for (int base = 0; base < words; base += kNumLongThreads) {
        const int w = base + threadIdx.x;
        const unsigned m0 = w < words ? bm_dense[w] : 0u;
        const int pc = __popc(m0);
        int incl = pc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        if (lane == 31) red[warp] = incl;
        __syncthreads();
        if (warp == 0) {
          int v = red[lane];
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
          }
          red[lane] = v;
        }
        __syncthreads();
        const int rtot = red[W - 1];
        int pos = off + (warp ? red[warp - 1] : 0) + incl - pc;
        unsigned m = m0;
        if (pos + pc > row_end) {  // more entries than the symbolic count: write nothing
          if (pc) atomicOr(err, ERR_COUNT);
          m = 0u;
        }
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1u;
          const int c = w0 + w * 32 + b;
          ccol[pos] = c;
          cval[pos] = __ldcg(acc + c);
          __stcg(acc + c, 0.0);
          ++pos;
        }
        off += rtot;
        __syncthreads();
      }
    }
    if (threadIdx.x == 0 && off != row_end) atomicOr(err, ERR_COUNT);
    ++rows_done;
  }
  if (redo && threadIdx.x == 0 && rows_done) atomicAdd(redo, rows_done);
}

// ---- dispatch ------------------------------------------------------------------------
template <int G, int LOG2T, bool OWNED, typename VT, bool COMP>
static cudaError_t run_num_group(const CsrDev &A, const CsrDev &B, const VT *av, const VT *bv,
                                 const int *crpt, int *ccol, double *cval, const int *rows,
                                 int count, int *err, CompArgs comp, cudaStream_t s) {
  using C = NumGroupCfg<G, LOG2T>;
  const void *f = (const void *)k_num_group<G, LOG2T, OWNED, VT, COMP>;
  const int grid = persistent_grid(f, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  k_num_group<G, LOG2T, OWNED, VT, COMP><<<grid, C::THREADS, C::SMEM, s>>>(
      A.rpt, A.col, av, B.rpt, B.col, bv, crpt, ccol, cval, rows, count, err, comp);
  return cudaGetLastError();
}

template <int G, bool OWNED, typename VT, bool COMP>
static cudaError_t num_group_bin(int bin, const CsrDev &A, const CsrDev &B, const VT *av,
                                 const VT *bv, const int *crpt, int *ccol, double *cval,
                                 const int *rows, int count, int *err, CompArgs comp,
                                 cudaStream_t s) {
#define NSPB_NG(L2T) \
  run_num_group<G, L2T, OWNED, VT, COMP>(A, B, av, bv, crpt, ccol, cval, rows, count, err, comp, s)
  switch (bin) {
    case 0: return NSPB_NG(5);
    case 1: return NSPB_NG(6);
    case 2: return NSPB_NG(7);
    case 3: return NSPB_NG(8);
    case 4: return NSPB_NG(9);
    default: return NSPB_NG(10);
  }
#undef NSPB_NG
}

template <int LOG2T, typename VT>
static cudaError_t run_num_block(const CsrDev &A, const CsrDev &B, const VT *av, const VT *bv,
                                 const int *crpt, int *ccol, double *cval, const int *rows,
                                 int count, int *err, int *redo, cudaStream_t s) {
  constexpr int T = 1 << LOG2T;
  const int smem = T * 12 + (T / 2) * 12 + (T / 2) * 4;
  const void *f = (const void *)k_num_block<LOG2T, VT>;
  const int grid = persistent_grid(f, kNumBlockThreads, smem, count, 1);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  k_num_block<LOG2T, VT><<<grid, kNumBlockThreads, smem, s>>>(
      A.rpt, A.col, av, B.rpt, B.col, bv, crpt, ccol, cval, rows, count, err, redo);
  return cudaGetLastError();
}

template <typename VT, bool COMP>
static cudaError_t numeric_bin_t(int bin, int lanes, bool owned, bool b_sorted, const CsrDev &A,
                                 const CsrDev &B, const VT *av, const VT *bv, const int *crpt,
                                 int *ccol, double *cval, const int *rows, int count, int *err,
                                 CompArgs comp, cudaStream_t s) {
  if (bin < kNumGroupBins) {
#define NSPB_GB(GL, OW) \
  num_group_bin<GL, OW, VT, COMP>(bin, A, B, av, bv, crpt, ccol, cval, rows, count, err, comp, s)
    if (owned) {
      if (lanes == 8) return NSPB_GB(8, true);
      if (lanes == 16) return NSPB_GB(16, true);
      return NSPB_GB(32, true);
    }
    if (lanes == 8) return NSPB_GB(8, false);
    if (lanes == 16) return NSPB_GB(16, false);
    return NSPB_GB(32, false);
#undef NSPB_GB
  }
  int *redo = COMP ? comp.redo : nullptr;
  switch (bin) {
    case kNumGroupBins:
      return run_num_block<11, VT>(A, B, av, bv, crpt, ccol, cval, rows, count, err, redo, s);
    case kNumGroupBins + 1:
      return run_num_block<12, VT>(A, B, av, bv, crpt, ccol, cval, rows, count, err, redo, s);
    case kNumGroupBins + 2:
      return run_num_block<13, VT>(A, B, av, bv, crpt, ccol, cval, rows, count, err, redo, s);
    default: {
      // dense accumulator per CTA when its footprint fits kDenseBudget,
      // else shared-memory column windows
      const int dsmem = kDenseWords * 4;
      const void *fd = (const void *)k_num_long_dense<VT>;
      int grid = persistent_grid(fd, kNumLongThreads, dsmem, count, 1);
      const long long per_cta = 8LL * (B.ncols > 0 ? B.ncols : 1);
      const long long fit = kDenseBudget / per_cta;
      if (grid > 0 && fit >= 1) {
        grid = (int)std::min<long long>(grid, fit);
        double *acc = nullptr;
        if (scratch_alloc(reinterpret_cast<void **>(&acc), (size_t)per_cta * grid, s) == NSPB_OK) {
          cudaError_t e = cudaMemsetAsync(acc, 0, (size_t)per_cta * grid, s);
          if (e == cudaSuccess) {
            k_num_long_dense<VT><<<grid, kNumLongThreads, dsmem, s>>>(
                A.rpt, A.col, av, B.rpt, B.col, bv, B.ncols, crpt, ccol, cval, rows, count, acc,
                err, redo);
            e = cudaGetLastError();
          }
          scratch_free(acc, s);
          return e;
        }
      }
      const int smem = kWin * 8 + kWinWords * 4;
      const void *f = (const void *)k_num_long<VT>;
      grid = persistent_grid(f, kNumLongThreads, smem, count, 1);
      if (grid <= 0) return cudaErrorInvalidConfiguration;
      k_num_long<VT><<<grid, kNumLongThreads, smem, s>>>(A.rpt, A.col, av, B.rpt, B.col, bv,
                                                         B.ncols, b_sorted, crpt, ccol, cval,
                                                         rows, count, err, redo);
      return cudaGetLastError();
    }
  }
}

cudaError_t launch_numeric_bin(int bin, int lanes, bool owned, bool b_sorted,
                               const CsrDev &A, const CsrDev &B, const int *crpt,
                               int *ccol, double *cval, const int *rows, int count,
                               int *err, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  return numeric_bin_t<double, false>(bin, lanes, owned, b_sorted, A, B, A.val, B.val, crpt,
                                      ccol, cval, rows, count, err, CompArgs{0, nullptr, nullptr},
                                      s);
}

cudaError_t launch_numeric_comp_bin(int bin, int lanes, bool owned, bool b_sorted,
                                    const CsrDev &A, const CsrDev &B, const int *crpt,
                                    int *ccol, double *cval, const int *rows, int count,
                                    int nmax, int *redo, int *max_deg, int *err,
                                    cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  return numeric_bin_t<float, true>(bin, lanes, owned, b_sorted, A, B, A.val32, B.val32, crpt,
                                    ccol, cval, rows, count, err, CompArgs{nmax, redo, max_deg},
                                    s);
}

}  // namespace nspb
