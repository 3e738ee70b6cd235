// Device-side building blocks shared by every kernel of the CSR product.
#pragma once

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "internal.h"

namespace cg = cooperative_groups;

namespace nspb {

// ---- operands of a row ---------------------------------------------------------
// The operands of global row r of a call and the row's index inside its
// product (see ProdTable in internal.h).
// MULTI false: one product, whose pointers stay kernel parameters (no
// registers held for them across the row); true: a table of products.
template <bool MULTI, typename VT>
__device__ __forceinline__ int prod_row(const ProdTable<VT> &t, int r, Operands<VT> &o) {
  if constexpr (!MULTI) {
    o = t.one;
    return r;
  } else {
    const int p = __ldg(t.prod_of_row + r);
    o = t.ops[p];
    return r - __ldg(t.row_off + p);
  }
}

// ---- error word bits (device -> host) ---------------------------------------
// A kernel never traps or spins forever: a bounded loop that runs out sets a
// bit here and the host turns it into NSPB_ERR_DEVICE.
enum : int {
  ERR_PROBE = 1,     // hash table probe sequence exhausted (table full)
  ERR_WAIT = 2,      // bounded wait in the single-pass scan ran out
  ERR_COUNT = 4,     // numeric row count differs from the symbolic count
  ERR_CAPACITY = 8   // a row exceeded the capacity of the kernel it was binned to
};

constexpr int kEmpty = -1;

// ---- bins ---------------------------------------------------------------------
// Symbolic rows are binned by ub = min(intprod, ncols(B)), the upper bound of
// their distinct columns; numeric rows by their exact nnz. Each bin names a
// kernel and a table size; see host launchers for the kernel of each bin.
constexpr int kSymBins = 12;  // 8 group tables 32..4096, 3 block tables 8K..32K, long
constexpr int kNumBins = 10;  // 6 group tables 32..1024, 3 block tables 2K..8K, long
constexpr int kSymGroupBins = 8;
constexpr int kNumGroupBins = 6;
constexpr int kSymLong = kSymBins - 1;
constexpr int kNumLong = kNumBins - 1;

// Inclusive upper limits of each bin (the last bin is unbounded). A symbolic
// bin of table size T = 32 << b takes rows with ub <= 0.75 T, so a row whose
// distinct columns reach its bound still leaves a quarter of the table free
// (linear probing slows sharply past that load).
__host__ __device__ constexpr int sym_limit(int b) {
  return b < kSymLong ? (24 << b) : 0x7fffffff;  // 24,48,...,24576
}
__host__ __device__ constexpr int num_limit(int b) {
  return b < kNumLong ? (16 << b) : 0x7fffffff;  // 16,32,...,4096
}
// Bins under runtime limits (BinLimits, the autotuner's thresholds).
__host__ __device__ __forceinline__ int sym_bin(int ub, const BinLimits &l) {
  int b = 0;
  while (b < kSymLong && ub > l.sym[b]) ++b;
  return b;
}
__host__ __device__ __forceinline__ int num_bin(int nz, const BinLimits &l) {
  int b = 0;
  while (b < kNumLong && nz > l.num[b]) ++b;
  return b;
}

// ---- hashing --------------------------------------------------------------------

// Fibonacci hashing: the HIGH bits of key*2^32/phi. Keys that differ by a
// multiple of a power of two (stencil planes n^2 apart) still spread, and runs
// of consecutive keys land on distinct shared-memory banks.
template <int LOG2T>
__device__ __forceinline__ unsigned hash_slot(int key) {
  return ((unsigned)key * 2654435769u) >> (32 - LOG2T);
}

__host__ __device__ constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }

// Streaming loads for data read once (A's entries): keep them out of L1.
__device__ __forceinline__ int ld_stream(const int *p) {
  int v;
  asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned ld_stream(const unsigned *p) {
  unsigned v;
  asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned ld_stream(const unsigned char *p) {
  unsigned short v;
  asm volatile("ld.global.nc.L1::no_allocate.u8 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_stream(const double *p) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// Probe sequences: linear (QUAD false: h, h+1, h+2, ...), best for the
// clustered columns of row groups; or triangular (QUAD true: h, h+1, h+3,
// h+6, ...), which breaks up clusters in the larger tables of block-per-row
// rows. Both visit every slot of a power-of-two table in its first 2^LOG2T
// probes.
//
// Symbolic insert of a key into an open-addressing table of 2^LOG2T int
// slots (empty = -1). Returns 1 when the key was new. The probe sequence is
// bounded by the table size.
template <int LOG2T, bool QUAD = false>
__device__ __forceinline__ int sym_insert(int *table, int key, int *err) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>(key);
#pragma unroll 1
  for (unsigned p = 0; p <= MASK; ++p) {
    const int cur = ((volatile int *)table)[h];
    if (cur == key) return 0;
    if (cur == kEmpty) {
      const int old = atomicCAS(table + h, kEmpty, key);
      if (old == kEmpty) return 1;
      if (old == key) return 0;
    }
    h = (h + (QUAD ? p : 0u) + 1u) & MASK;
  }
  atomicOr(err, ERR_PROBE);
  return 0;
}

// Numeric insert-accumulate into (keys, vals). With OWNED the caller
// guarantees that no other thread touches the same key until the next group
// barrier, so the value update is a plain read-modify-write and the sum of
// each entry is formed in the caller's step order (deterministic). Without
// OWNED the value is added atomically.
template <int LOG2T, bool OWNED, bool QUAD = false>
__device__ __forceinline__ void num_insert(int *keys, double *vals, int key,
                                           double p, int *err) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>(key);
#pragma unroll 1
  for (unsigned q = 0; q <= MASK; ++q) {
    const int cur = ((volatile int *)keys)[h];
    bool hit = cur == key;
    if (!hit && cur == kEmpty) {
      const int old = atomicCAS(keys + h, kEmpty, key);
      hit = (old == kEmpty) || (old == key);
    }
    if (hit) {
      if (OWNED) {
        vals[h] = __dadd_rn(vals[h], p);
      } else {
        atomicAdd(vals + h, p);
      }
      return;
    }
    h = (h + (QUAD ? q : 0u) + 1u) & MASK;
  }
  atomicOr(err, ERR_PROBE);
}

// Slot of `key` in (keys), inserting it when absent; -1 (and the error word)
// when the probe sequence is exhausted.
template <int LOG2T, bool QUAD = false>
__device__ __forceinline__ int num_slot(int *keys, int key, int *err) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>(key);
#pragma unroll 1
  for (unsigned q = 0; q <= MASK; ++q) {
    const int cur = ((volatile int *)keys)[h];
    if (cur == key) return (int)h;
    if (cur == kEmpty) {
      const int old = atomicCAS(keys + h, kEmpty, key);
      if (old == kEmpty || old == key) return (int)h;
    }
    h = (h + (QUAD ? q : 0u) + 1u) & MASK;
  }
  atomicOr(err, ERR_PROBE);
  return -1;
}

// Error-free fp32 accumulation of a*b into the pair (s, c): TwoProduct by FMA,
// then TwoSum of s and the high part; the low parts go to c. Rounding is
// explicit so no step is contracted or reordered.
__device__ __forceinline__ void comp_add(float2 &sc, float a, float b) {
  const float ph = __fmul_rn(a, b);
  const float pl = __fmaf_rn(a, b, -ph);
  const float t = __fadd_rn(sc.x, ph);
  const float z = __fsub_rn(t, sc.x);
  const float e = __fadd_rn(__fsub_rn(sc.x, __fsub_rn(t, z)), __fsub_rn(ph, z));
  sc.x = t;
  sc.y = __fadd_rn(sc.y, __fadd_rn(e, pl));
}

// Value loads as fp64 from fp64 or fp32 arrays (fp32 products are then exact
// in fp64: 24 + 24 significant bits).
__device__ __forceinline__ double ldv(const double *p) { return __ldg(p); }
__device__ __forceinline__ double ldv(const float *p) { return (double)__ldg(p); }
__device__ __forceinline__ double ldv_stream(const double *p) { return ld_stream(p); }
__device__ __forceinline__ double ldv_stream(const float *p) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return (double)v;
}

// Shared state of row_products: a queue of one round's A entries {B row
// start, B row end, A value as two ints} and two sets of counters {medium
// entries, long entries, medium cursor}, used in alternate rounds so that one
// set is cleared while the other is in use. Counters start at zero.
template <int THREADS>
struct RowQueue {
  int4 q[THREADS];
  int ctr[2][3];
};

template <int THREADS>
__device__ __forceinline__ void row_queue_init(RowQueue<THREADS> &rq) {
  if (threadIdx.x < 6) (&rq.ctr[0][0])[threadIdx.x] = 0;
}

// Every product of one A row, spread evenly over a block of THREADS threads
// whatever the lengths of the B rows it touches (power-law matrices mix rows
// of one entry with hub rows of 10^4 and more). The A row is taken in rounds
// of THREADS entries, one per thread:
//   - a B row of at most kRowSmall entries (4 when the round holds fewer than
//     THREADS/4 entries) is walked by its thread, four entries' loads at a
//     time: up to THREADS independent gather chains in flight;
//   - a longer B row goes to a queue; warps take queued rows one at a time
//     from a shared cursor, lanes over the row's entries;
//   - a B row of THREADS entries or more is walked by the whole block, thread
//     t taking the products whose index in the round's concatenation of such
//     rows is t mod THREADS.
// f(c, a, b) gets the B entry's column, the A value and the B value (values 0
// when aval / bval are null). Every thread of the block must call this with
// the same (a0, a1) after a block barrier, and a block barrier must separate
// two calls.
#ifndef NSPB_ROW_SMALL
#define NSPB_ROW_SMALL 16
#endif
constexpr int kRowSmall = NSPB_ROW_SMALL;  // longest B row one thread walks alone

template <int THREADS, typename VT, typename F>
__device__ __forceinline__ void row_products(const int *__restrict__ acol,
                                             const VT *__restrict__ aval,
                                             const int *__restrict__ brpt,
                                             const int *__restrict__ bcol,
                                             const VT *__restrict__ bval, int a0, int a1,
                                             RowQueue<THREADS> &rq, F &&f) {
  static_assert((THREADS & (THREADS - 1)) == 0, "THREADS must be a power of two");
  const int lane = threadIdx.x & 31;
  auto bv = [&](int e) -> double { return bval ? ldv(bval + e) : 0.0; };
  // entries [e, end) with stride S, two loads in flight per thread
  auto strided = [&](int e, int end, double a, auto S) {
    constexpr int kS = decltype(S)::value;
    for (; e + kS < end; e += 2 * kS) {
      const int c0 = __ldg(bcol + e), c1 = __ldg(bcol + e + kS);
      const double b0 = bv(e), b1 = bv(e + kS);
      f(c0, a, b0);
      f(c1, a, b1);
    }
    if (e < end) f(__ldg(bcol + e), a, bv(e));
  };
  int par = 0;
  for (int jr = a0; jr < a1; jr += THREADS, par ^= 1) {  // uniform across the block
    const int small_max = min(THREADS, a1 - jr) * 4 >= THREADS ? kRowSmall : 4;
    const int j = jr + (int)threadIdx.x;
    if (j < a1) {
      const int k = ld_stream(acol + j);
      const double a = aval ? ldv_stream(aval + j) : 0.0;
      const int s0 = __ldg(brpt + k), s1 = __ldg(brpt + k + 1);
      if (s1 - s0 <= small_max) {
        int e = s0;
        for (; e + 4 <= s1; e += 4) {
          const int c0 = __ldg(bcol + e), c1 = __ldg(bcol + e + 1);
          const int c2 = __ldg(bcol + e + 2), c3 = __ldg(bcol + e + 3);
          const double b0 = bv(e), b1 = bv(e + 1), b2 = bv(e + 2), b3 = bv(e + 3);
          f(c0, a, b0);
          f(c1, a, b1);
          f(c2, a, b2);
          f(c3, a, b3);
        }
        for (; e < s1; ++e) f(__ldg(bcol + e), a, bv(e));
      } else {
        const int big = (s1 - s0 >= THREADS) ? 1 : 0;
        const int slot = atomicAdd(&rq.ctr[par][big], 1);
        rq.q[big ? THREADS - 1 - slot : slot] =
            make_int4(s0, s1, __double2loint(a), __double2hiint(a));
      }
    }
    __syncthreads();
    // the other counter set was last read before the previous round's closing
    // barrier and is next written after this round's
    if (threadIdx.x == 0) rq.ctr[par ^ 1][0] = rq.ctr[par ^ 1][1] = rq.ctr[par ^ 1][2] = 0;
    const int nm = rq.ctr[par][0], nb = rq.ctr[par][1];
    for (;;) {
      int i = 0;
      if (lane == 0) i = atomicAdd(&rq.ctr[par][2], 1);
      i = __shfl_sync(0xffffffffu, i, 0);
      if (i >= nm) break;
      const int4 v = rq.q[i];
      strided(v.x + lane, v.y, __hiloint2double(v.w, v.z), std::integral_constant<int, 32>());
    }
    unsigned pos = 0;  // products of the long rows before row i, mod 2^32
    for (int i = 0; i < nb; ++i) {
      const int4 v = rq.q[THREADS - 1 - i];
      const int first = (int)((threadIdx.x - pos) & (unsigned)(THREADS - 1));
      strided(v.x + first, v.y, __hiloint2double(v.w, v.z),
              std::integral_constant<int, THREADS>());
      pos += (unsigned)(v.y - v.x);
    }
    __syncthreads();
  }
  // counters of the last round (the other set was cleared during it); the
  // caller's barrier before the next call orders this
  if (a1 > a0 && threadIdx.x == 0)
    rq.ctr[par ^ 1][0] = rq.ctr[par ^ 1][1] = rq.ctr[par ^ 1][2] = 0;
}

// Intermediate products of one A row and the range of columns they can
// reach: [lo, hi] from the first and last entries of the B rows it touches
// when B's rows are sorted, else [0, ncols). Empty rows give lo > hi.
struct RowSpan {
  long long ip;
  int lo, hi;
};

template <int THREADS>
struct SpanScratch {
  long long ip[THREADS / 32];
  int lo[THREADS / 32], hi[THREADS / 32];
};

// Block-wide; every thread gets the row's span. Ends with a block barrier
// and reads sc after it, so a block barrier must come before the next call.
template <int THREADS>
__device__ __forceinline__ RowSpan row_span(const int *__restrict__ acol,
                                            const int *__restrict__ brpt,
                                            const int *__restrict__ bcol, int a0, int a1,
                                            bool b_sorted, int ncols, SpanScratch<THREADS> &sc) {
  constexpr int W = THREADS / 32;
  long long ip = 0;
  int lo = 0x7fffffff, hi = -1;
  for (int j = a0 + (int)threadIdx.x; j < a1; j += THREADS) {
    const int k = __ldg(acol + j);
    const int s0 = __ldg(brpt + k), s1 = __ldg(brpt + k + 1);
    if (s1 > s0) {
      ip += s1 - s0;
      if (b_sorted) {
        lo = min(lo, __ldg(bcol + s0));
        hi = max(hi, __ldg(bcol + s1 - 1));
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ip += __shfl_xor_sync(0xffffffffu, ip, o);
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sc.ip[warp] = ip;
    sc.lo[warp] = lo;
    sc.hi[warp] = hi;
  }
  __syncthreads();
  RowSpan r{0, 0x7fffffff, -1};
#pragma unroll
  for (int w = 0; w < W; ++w) {
    r.ip += sc.ip[w];
    r.lo = min(r.lo, sc.lo[w]);
    r.hi = max(r.hi, sc.hi[w]);
  }
  if (!b_sorted && r.ip > 0) {
    r.lo = 0;
    r.hi = ncols - 1;
  }
  // columns outside [0, ncols) fall outside every window and are dropped
  r.lo = max(r.lo, 0);
  r.hi = min(r.hi, ncols - 1);
  return r;
}

// Next row index of a block-per-row kernel from a launch-wide ticket counter
// (zero at launch): rows go to blocks as they free up, so a block that drew a
// heavy row draws no more meanwhile. Returns count when none is left.
__device__ __forceinline__ int next_row(int *ticket, int count, int *s_slot) {
  __syncthreads();  // every thread has read the previous slot value
  if (threadIdx.x == 0) *s_slot = atomicAdd(ticket, 1);
  __syncthreads();
  const int r = *s_slot;
  return r < count ? r : count;
}

// Entry-map layout (k_sym_map writes, k_num_map reads): four consecutive
// steps of a chunk form a quad, stored as one 4-byte word per lane, when each
// of their B rows fits the group of G lanes and they hold at least 3G
// products (so the words waste at most a quarter of their bytes).
template <int G>
__device__ __forceinline__ bool map_quad(const int (&len)[4]) {
  return len[0] <= G && len[1] <= G && len[2] <= G && len[3] <= G &&
         len[0] + len[1] + len[2] + len[3] >= 3 * G;
}

// Monotone bucket map of a key in [lo, lo+range) onto [0, nb): used to sort
// the entries of one row (bucket scatter, then rank inside each bucket).
__device__ __forceinline__ int bucket_of(int key, int lo, float scale, int nb) {
  int b = (int)((float)(key - lo) * scale);
  return b < nb - 1 ? b : nb - 1;
}

// True when B rows k and kt are one run of shifted rows (bit k of bits: B row k is row k-1 moved by one
// column shift; launch_brow_shift);
// runs are only followed over 31 rows at most (false beyond).
__device__ __forceinline__ bool same_run(const unsigned *__restrict__ bits, int k, int kt) {
  if (k == kt) return true;
  const int lo = min(k, kt) + 1, hi = max(k, kt);
  if (hi - lo >= 31) return false;
  const int wa = lo >> 5, wb = hi >> 5;
  const unsigned ma = 0xffffffffu << (lo & 31);
  const unsigned mb = 0xffffffffu >> (31 - (hi & 31));
  if (wa == wb) return (__ldg(bits + wa) & (ma & mb)) == (ma & mb);
  return (__ldg(bits + wa) & ma) == ma && (__ldg(bits + wb) & mb) == mb;
}

}  // namespace nspb
