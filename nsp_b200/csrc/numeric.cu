// Numeric phase: values of C, columns ascending within each row.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu):
//   nsp_calculate_value_col_bin_mpwarp     :1307-1401 (4/8/16 threads per row)
//   nsp_calculate_value_col_bin_each_warp  :1405-1494
//   nsp_calculate_value_col_bin_each_tb    :1499-1627 (block per row)
//   ..._each_tb_outsort + nsp_calc_val_sort_rows  :1632-1714,
//                                          nsp_calc_val_sort_rows.cu:24-527
//   ..._chunk_dynamic / nsp_calc_C_dense / ..._chunk_B_dense :1725-2151
// The reference sorts each row by an O(nnz^2) rank count. Here each row of up
// to 4096 entries is sorted by a monotone bucket scatter over [min col, max
// col] followed by a rank count inside each bucket, in shared memory, and
// written coalesced; longer rows need no sort at all: a bitmap of their
// columns gives each column its output position (k_num_rank).
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

// VT: value type of A and B (double, or float in the compensated mode).
// COMP: fp32 inputs with the error-free pair accumulation for short rows.
template <int G, int LOG2T, bool OWNED, typename VT, bool COMP, bool MULTI>
__global__ void __launch_bounds__(256)
    k_num_group(const ProdTable<VT> src, const int *__restrict__ crpt, int *__restrict__ ccol,
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
    // 16-byte stores: two values or four keys each (both arrays start on a
    // 16-byte boundary)
#pragma unroll 4
    for (int s = lane; s < C::T / 2; s += G)
      reinterpret_cast<double2 *>(vals)[s] = make_double2(0.0, 0.0);
#pragma unroll 2
    for (int s = lane; s < C::T / 4; s += G)
      reinterpret_cast<int4 *>(keys)[s] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    tile.sync();
    Operands<VT> op;
    const int lr = prod_row<MULTI>(src, row, op);
    const int *acol = op.acol, *brpt = op.brpt, *bcol = op.bcol;
    const VT *aval = op.aval, *bval = op.bval;
    const int a0 = op.arpt[lr], a1 = op.arpt[lr + 1];
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
    for (int b = lane; b < C::NB / 4; b += G) reinterpret_cast<int4 *>(cnt)[b] = make_int4(0, 0, 0, 0);
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
    // C is written once and not read here again: streaming (evict-first)
    // stores leave L2 to the B rows the next rows gather
    for (int q = lane; q < n; q += G) {
      __stcs(ccol + c0 + q, keys[q]);
      __stcs(cval + c0 + q, vals[q]);
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

// Blocks per SM that the shared memory of a block-per-row kernel admits, given
// to __launch_bounds__ as the minimum so that ptxas budgets registers for that
// many blocks: without it ptxas kept these kernels at 32 registers a thread
// (the budget of 2048 resident threads) and spilled, 290 bytes a thread in
// k_num_rank, while their shared memory holds one or two blocks per SM.
// k_num_block needs 20 bytes per table slot: 2^13 slots admit one block,
// 2^12 two, smaller tables four (2048 threads).
__host__ __device__ constexpr int num_block_minb(int log2t) {
  return log2t >= 13 ? 1 : log2t == 12 ? 2 : 4;
}

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

template <int LOG2T, typename VT, bool MULTI>
__global__ void __launch_bounds__(kNumBlockThreads, num_block_minb(LOG2T))
    k_num_block(const ProdTable<VT> src, const int *__restrict__ crpt, int *__restrict__ ccol,
                double *__restrict__ cval, const int *__restrict__ rows, int count,
                int *__restrict__ err, int *__restrict__ redo, int *__restrict__ ticket) {
  constexpr int T = 1 << LOG2T, H = T / 2, NB = T / 2;
  constexpr int PER = NB / kNumBlockThreads;
  extern __shared__ __align__(16) unsigned char smem_num[];
  double *vals = reinterpret_cast<double *>(smem_num);
  double *bvals = vals + T;
  int *keys = reinterpret_cast<int *>(bvals + H);
  int *bkeys = keys + T;
  int *cnt = bkeys + H;
  __shared__ int red[kNumBlockThreads / 32];
  __shared__ int s_mn, s_mx, s_slot;
  __shared__ RowQueue<kNumBlockThreads> rq;
  row_queue_init(rq);
  const int lane = threadIdx.x & 31;
  int rows_done = 0;
  for (int r = next_row(ticket, count, &s_slot); r < count; r = next_row(ticket, count, &s_slot)) {
    const int row = rows ? rows[r] : r;
    // 16-byte stores (vals, keys and cnt start on 16-byte boundaries)
    for (int s = threadIdx.x; s < T / 2; s += kNumBlockThreads)
      reinterpret_cast<double2 *>(vals)[s] = make_double2(0.0, 0.0);
    for (int s = threadIdx.x; s < T / 4; s += kNumBlockThreads)
      reinterpret_cast<int4 *>(keys)[s] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    for (int b = threadIdx.x; b < NB / 4; b += kNumBlockThreads)
      reinterpret_cast<int4 *>(cnt)[b] = make_int4(0, 0, 0, 0);
    if (threadIdx.x == 0) {
      s_mn = 0x7fffffff;
      s_mx = -1;
    }
    __syncthreads();
    Operands<VT> op;
    const int lr = prod_row<MULTI>(src, row, op);
    const int a0 = op.arpt[lr], a1 = op.arpt[lr + 1];
    int mn = 0x7fffffff, mx = -1;
    row_products<kNumBlockThreads>(op.acol, op.aval, op.brpt, op.bcol, op.bval, a0, a1, rq,
                                   [&](int key, double a, double b) {
      num_insert<LOG2T, false, true>(keys, vals, key, __dmul_rn(a, b), err);
      mn = min(mn, key);
      mx = max(mx, key);
    });
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
      __stcs(ccol + c0 + q, keys[q]);
      __stcs(cval + c0 + q, vals[q]);
    }
    __syncthreads();
  }
  if (redo && threadIdx.x == 0 && rows_done) atomicAdd(redo, rows_done);
}

// ---- rows of more than 4096 entries: column ranks from a row bitmap -----------
// A first pass over the row's products sets its distinct columns as bits of a
// shared-memory bitmap over the row's column span [lo, hi] (see row_span). A
// prefix count of the bitmap then gives every column its rank, which is its
// position in the sorted output row: the columns are written in order with no
// sort, and a second pass adds each product straight into its output slot,
// in shared memory when the row has at most kRankVals entries, else with fp64
// atomics into the row's part of C.val (which stays in L2 while the row is
// built: 8 bytes per entry). A span wider than 2^20 columns is covered in
// windows of 2^20, each with its own two passes.
//
// Thread t owns the 64-bit words [t*per, (t+1)*per) of a window's bitmap, so
// warp w owns 32*per words; the rank of column c is base[warp of c] +
// pre[c/64] + the bits below c in its word, pre[] being the 16-bit count
// inside the warp's words (at most 511*64 bits precede a word there).
constexpr int kRankThreads = 1024;
constexpr int kRankVals = 6144;          // 48 KB of fp64 accumulators
constexpr int kRankMaxCols = 1 << 20;    // bitmap of 2^14 64-bit words, 128 KB
#ifndef NSPB_RANK_FROM_BIN
#define NSPB_RANK_FROM_BIN kNumLong
#endif
constexpr int kRankFromBin = NSPB_RANK_FROM_BIN;  // first numeric bin sent here

// log2 of the 64-bit words per thread for a window of `cols` columns
__host__ __device__ inline int rank_per_log2(int cols) {
  int pl = 0;
  while (pl < 4 && (kRankThreads << (pl + 6)) < cols) ++pl;
  return pl;
}
__host__ __device__ constexpr int rank_smem(int per_log2) {
  return (kRankThreads << per_log2) * 10 + kRankVals * 8;
}

// Blocks per SM the rank kernel's shared memory admits for the widest window:
// windows of 2^19 columns or more (per_log2 >= 3, 131 KB and up) leave room for
// one block, which may then use 64 registers a thread; narrower ones for two.
__host__ __device__ constexpr int rank_minb(int per_log2) { return per_log2 >= 3 ? 1 : 2; }

// C.val slices of rows longer than the shared value buffer are zero-filled
// and then added into, product by product, while the walk gathers B rows that
// do not fit in L2 beside them. An evict-last L2 policy on those stores and
// adds keeps the slices resident between the two, instead of their lines
// being written back and fetched again for the adds (power-law 1M product
// 17.68 -> 16.00 ms).
__device__ __forceinline__ unsigned long long l2_evict_last_policy() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void st_global_keep(double *p, double v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(__cvta_generic_to_global(p)),
               "d"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void red_add_global_keep(double *p, double v, unsigned long long pol) {
  asm volatile("red.global.add.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(__cvta_generic_to_global(p)),
               "d"(v), "l"(pol)
               : "memory");
}

template <typename VT, int MINB, bool MULTI>
__global__ void __launch_bounds__(kRankThreads, MINB)
    k_num_rank(const ProdTable<VT> src, int b_sorted, int pl_max, const int *__restrict__ crpt,
               int *__restrict__ ccol, double *__restrict__ cval,
               const int *__restrict__ rows, int count, int *__restrict__ err,
               int *__restrict__ redo, int *__restrict__ ticket) {
  extern __shared__ __align__(16) unsigned long long bm64[];
  const int max_words = kRankThreads << pl_max;
  unsigned *bm32 = reinterpret_cast<unsigned *>(bm64);
  unsigned short *pre = reinterpret_cast<unsigned short *>(bm64 + max_words);
  double *vals = reinterpret_cast<double *>(pre + max_words);  // max_words*2: multiple of 8
  __shared__ int base[kRankThreads / 32];
  __shared__ int s_total, s_slot;
  __shared__ RowQueue<kRankThreads> rq;
  __shared__ SpanScratch<kRankThreads> sc;
  row_queue_init(rq);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int rows_done = 0;
  for (int q = threadIdx.x; q < max_words; q += kRankThreads) bm64[q] = 0ull;
  for (int r = next_row(ticket, count, &s_slot); r < count; r = next_row(ticket, count, &s_slot)) {
    const int row = rows ? rows[r] : r;
    Operands<VT> op;
    const int lr = prod_row<MULTI>(src, row, op);
    const int *acol = op.acol, *brpt = op.brpt, *bcol = op.bcol;
    const VT *aval = op.aval, *bval = op.bval;
    const int ncols = op.ncols;
    const int a0 = op.arpt[lr], a1 = op.arpt[lr + 1];
    const int row_end = crpt[row + 1];
    int off = crpt[row];
    bool bad = false;  // block-uniform
    const RowSpan sp = row_span<kRankThreads>(acol, brpt, bcol, a0, a1, b_sorted != 0, ncols, sc);
    for (long long wl = sp.lo; wl <= sp.hi; wl += kRankMaxCols) {
      const int w0 = (int)wl;
      const int wn = (int)min((long long)kRankMaxCols, (long long)sp.hi - wl + 1);
      const int pl = rank_per_log2(wn);
      const int per = 1 << pl;
      const int t0 = threadIdx.x << pl;  // this thread's first word
      // pass 1: distinct columns of the window
      row_products<kRankThreads>(acol, (const VT *)nullptr, brpt, bcol, (const VT *)nullptr, a0,
                                 a1, rq, [&](int c, double, double) {
        const unsigned d = (unsigned)(c - w0);
        if (d < (unsigned)wn) {
          const unsigned bit = 1u << (d & 31u);
          if (!(bm32[d >> 5] & bit)) atomicOr(bm32 + (d >> 5), bit);
        }
      });
      __syncthreads();
      // ranks: counts of this thread's words, scanned over the warp and the block
      int cnt = 0;
      for (int i = 0; i < per; ++i) cnt += __popcll(bm64[t0 + i]);
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) base[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        const int t = base[lane];
        int v = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        base[lane] = v - t;
        if (lane == 31) s_total = v;
      }
      __syncthreads();
      const int total = s_total;
      if (!bad && off + total > row_end) {  // more columns than the symbolic count
        bad = true;
        if (threadIdx.x == 0) atomicOr(err, ERR_COUNT);
      }
      const bool in_smem = total <= kRankVals;
      {
        int p = incl - cnt;
        int pos = off + base[warp] + p;
        for (int i = 0; i < per; ++i) {
          const int w = t0 + i;
          unsigned long long m = bm64[w];
          pre[w] = (unsigned short)p;
          p += __popcll(m);
          if (bad) continue;
          while (m) {
            const int b = __ffsll((long long)m) - 1;
            m &= m - 1ull;
            __stcs(ccol + pos++, w0 + (w << 6) + b);
          }
        }
      }
      if (!bad) {
        if (in_smem) {
          for (int i = threadIdx.x; i < total; i += kRankThreads) vals[i] = 0.0;
        } else {
          const unsigned long long pol = l2_evict_last_policy();
          for (int i = threadIdx.x; i < total; i += kRankThreads)
            st_global_keep(cval + off + i, 0.0, pol);
        }
      }
      __syncthreads();
      // pass 2: values into their ranks
      if (!bad) {
        const int shift = 5 + pl;
        auto rank_of = [&](unsigned d) {
          const int w = (int)(d >> 6);
          return base[w >> shift] + pre[w] + __popcll(bm64[w] & ((1ull << (d & 63u)) - 1ull));
        };
        if (in_smem) {
          row_products<kRankThreads>(acol, aval, brpt, bcol, bval, a0, a1, rq,
                                     [&](int c, double a, double b) {
            const unsigned d = (unsigned)(c - w0);
            if (d < (unsigned)wn) atomicAdd(vals + rank_of(d), __dmul_rn(a, b));
          });
        } else {
          double *dst = cval + off;
          const unsigned long long pol = l2_evict_last_policy();
          row_products<kRankThreads>(acol, aval, brpt, bcol, bval, a0, a1, rq,
                                     [&](int c, double a, double b) {
            const unsigned d = (unsigned)(c - w0);
            if (d < (unsigned)wn) red_add_global_keep(dst + rank_of(d), __dmul_rn(a, b), pol);
          });
        }
      }
      __syncthreads();
      if (in_smem && !bad)
        for (int i = threadIdx.x; i < total; i += kRankThreads) __stcs(cval + off + i, vals[i]);
      for (int i = 0; i < per; ++i) bm64[t0 + i] = 0ull;
      off += total;
      __syncthreads();  // bitmap clear and value copy-out before the next window
    }
    if (!bad && off != row_end && threadIdx.x == 0) atomicOr(err, ERR_COUNT);
    ++rows_done;  // compensated mode: every row here is an fp64 row
  }
  if (redo && threadIdx.x == 0 && rows_done) atomicAdd(redo, rows_done);
}

template <typename VT>
static cudaError_t run_num_rank(const ProdTable<VT> &t, const ProdInfo &info, bool b_sorted,
                                const int *crpt, int *ccol, double *cval, const int *rows,
                                int count, int *err, int *redo, int *ticket, cudaStream_t s) {
  const int pl = rank_per_log2((int)std::min<long long>(info.max_ncols, kRankMaxCols));
  const int smem = rank_smem(pl);
  const bool multi = t.prod_of_row != nullptr;
  auto kern = rank_minb(pl) == 1 ? (multi ? k_num_rank<VT, 1, true> : k_num_rank<VT, 1, false>)
                                 : (multi ? k_num_rank<VT, 2, true> : k_num_rank<VT, 2, false>);
  const int grid = persistent_grid((const void *)kern, kRankThreads, smem, count, 1);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, kRankThreads, smem, s>>>(t, b_sorted ? 1 : 0, pl, crpt, ccol, cval, rows, count,
                                        err, redo, ticket);
  return cudaGetLastError();
}

// ---- dispatch ------------------------------------------------------------------------
template <int G, int LOG2T, bool OWNED, typename VT, bool COMP>
static cudaError_t run_num_group(const ProdTable<VT> &t, const int *crpt, int *ccol,
                                 double *cval, const int *rows, int count, int *err,
                                 CompArgs comp, cudaStream_t s) {
  using C = NumGroupCfg<G, LOG2T>;
  auto kern = t.prod_of_row ? k_num_group<G, LOG2T, OWNED, VT, COMP, true>
                            : k_num_group<G, LOG2T, OWNED, VT, COMP, false>;
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(t, crpt, ccol, cval, rows, count, err, comp);
  return cudaGetLastError();
}

template <int G, bool OWNED, typename VT, bool COMP>
static cudaError_t num_group_bin(int bin, const ProdTable<VT> &t, const int *crpt, int *ccol,
                                 double *cval, const int *rows, int count, int *err,
                                 CompArgs comp, int tshift, cudaStream_t s) {
#define NSPB_NG(L2T) \
  run_num_group<G, L2T, OWNED, VT, COMP>(t, crpt, ccol, cval, rows, count, err, comp, s)
  // bin b holds rows of at most 16 << b entries; its table has 32 << (b + tshift)
  // slots (load <= 1/2 or 1/4), 1024 at most
  switch (std::min(5 + bin + tshift, 10)) {
    case 5: return NSPB_NG(5);
    case 6: return NSPB_NG(6);
    case 7: return NSPB_NG(7);
    case 8: return NSPB_NG(8);
    case 9: return NSPB_NG(9);
    default: return NSPB_NG(10);
  }
#undef NSPB_NG
}

template <int LOG2T, typename VT>
static cudaError_t run_num_block(const ProdTable<VT> &t, const int *crpt, int *ccol,
                                 double *cval, const int *rows, int count, int *err, int *redo,
                                 int *ticket, cudaStream_t s) {
  constexpr int T = 1 << LOG2T;
  const int smem = T * 12 + (T / 2) * 12 + (T / 2) * 4;
  auto kern = t.prod_of_row ? k_num_block<LOG2T, VT, true> : k_num_block<LOG2T, VT, false>;
  const int grid = persistent_grid((const void *)kern, kNumBlockThreads, smem, count, 1);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, kNumBlockThreads, smem, s>>>(t, crpt, ccol, cval, rows, count, err, redo, ticket);
  return cudaGetLastError();
}

template <typename VT, bool COMP>
static cudaError_t numeric_bin_t(int bin, int lanes, bool owned, bool b_sorted,
                                 const ProdTable<VT> &t, const ProdInfo &info, const int *crpt,
                                 int *ccol, double *cval, const int *rows, int count, int *err,
                                 CompArgs comp, int *ticket, int tshift, cudaStream_t s) {
  if (bin < kNumGroupBins) {
#define NSPB_GB(GL, OW) \
  num_group_bin<GL, OW, VT, COMP>(bin, t, crpt, ccol, cval, rows, count, err, comp, tshift, s)
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
  if (bin >= kRankFromBin)
    return run_num_rank<VT>(t, info, b_sorted, crpt, ccol, cval, rows, count, err, redo,
                            ticket, s);
  switch (bin) {
    case kNumGroupBins:
      return run_num_block<11, VT>(t, crpt, ccol, cval, rows, count, err, redo, ticket, s);
    case kNumGroupBins + 1:
      return run_num_block<12, VT>(t, crpt, ccol, cval, rows, count, err, redo, ticket, s);
    default:
      return run_num_block<13, VT>(t, crpt, ccol, cval, rows, count, err, redo, ticket, s);
  }
}

cudaError_t launch_numeric_bin(int bin, int lanes, bool owned, bool b_sorted,
                               const ProdTable<double> &t, const ProdInfo &info,
                               const int *crpt, int *ccol, double *cval, const int *rows,
                               int count, int *err, int *ticket, int tshift, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  return numeric_bin_t<double, false>(bin, lanes, owned, b_sorted, t, info, crpt, ccol, cval,
                                      rows, count, err, CompArgs{0, nullptr, nullptr}, ticket,
                                      tshift, s);
}

cudaError_t launch_numeric_comp_bin(int bin, int lanes, bool owned, bool b_sorted,
                                    const ProdTable<float> &t, const ProdInfo &info,
                                    const int *crpt, int *ccol, double *cval, const int *rows,
                                    int count, int nmax, int *redo, int *max_deg, int *err,
                                    int *ticket, int tshift, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  return numeric_bin_t<float, true>(bin, lanes, owned, b_sorted, t, info, crpt, ccol, cval, rows,
                                    count, err, CompArgs{nmax, redo, max_deg}, ticket, tshift,
                                    s);
}

}  // namespace nspb
