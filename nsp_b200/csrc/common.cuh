// Device-side building blocks shared by every kernel of the CSR product.
#pragma once

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cg = cooperative_groups;

namespace nspb {

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
__host__ __device__ __forceinline__ int sym_bin(int ub) {
  int b = 0;
  while (b < kSymLong && ub > sym_limit(b)) ++b;
  return b;
}
__host__ __device__ __forceinline__ int num_bin(int nz) {
  int b = 0;
  while (b < kNumLong && nz > num_limit(b)) ++b;
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
__device__ __forceinline__ double ld_stream(const double *p) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// Symbolic insert of a key into an open-addressing table of 2^LOG2T int
// slots (empty = -1). Returns 1 when the key was new. The probe sequence is
// bounded by the table size.
template <int LOG2T>
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
    h = (h + 1u) & MASK;
  }
  atomicOr(err, ERR_PROBE);
  return 0;
}

// Numeric insert-accumulate into (keys, vals). With OWNED the caller
// guarantees that no other thread touches the same key until the next group
// barrier, so the value update is a plain read-modify-write and the sum of
// each entry is formed in the caller's step order (deterministic). Without
// OWNED the value is added atomically.
template <int LOG2T, bool OWNED>
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
    h = (h + 1u) & MASK;
  }
  atomicOr(err, ERR_PROBE);
}

// Slot of `key` in (keys), inserting it when absent; -1 (and the error word)
// when the probe sequence is exhausted.
template <int LOG2T>
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
    h = (h + 1u) & MASK;
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

// Padded index of a bucket counter: one spare slot per 32 counters, so a
// lane that owns a run of consecutive counters hits its own bank.
__device__ __forceinline__ int cpad(int b) { return b + (b >> 5); }

// Monotone bucket map of a key in [lo, lo+range) onto [0, nb): used to sort
// the entries of one row (bucket scatter, then rank inside each bucket).
__device__ __forceinline__ int bucket_of(int key, int lo, float scale, int nb) {
  int b = (int)((float)(key - lo) * scale);
  return b < nb - 1 ? b : nb - 1;
}

}  // namespace nspb
