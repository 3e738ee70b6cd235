// Staged-walk numeric kernels of the row-group bins: rows of at most 512
// entries whose B rows are strictly increasing, one lane group a row. The
// host takes them when the rows compress (at least 1.5 intermediate products
// per entry of C); otherwise numeric.cu's hash-sort kernels run.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu):
//   nsp_calculate_value_col_bin_mpwarp / _each_warp :1307-1494 (shared-memory
//   hash with atomic adds, then an O(nnz^2) rank sort)
//
// Shape of one row (a lane group of G lanes, G = 8, 16 or 32):
//   - the A row is taken G entries at a time; each lane stages one entry's
//     {B row start, B row end, A value} in shared memory, so every step reads
//     its B row bounds with one broadcast load;
//   - D B rows at a time have their columns and values loaded before the
//     first of them is inserted (loads in flight while the table is updated);
//   - a step covers one B row, a lane per entry; its key is looked up at its
//     home slot first, and only a miss enters the probe loop (a 4x-load table
//     makes almost every step of a stencil row collision-free);
//   - values are not cleared between rows; the lane that inserts a key writes
//     0 + a*b, later steps add in A-row order (deterministic, bit for bit the
//     oracle's sum);
//   - the row is sorted by a bucket counting sort whose monotone map spans
//     [first column, last column] of the row, taken from the ends of the
//     (sorted) B rows while staging; the compaction of the table counts the
//     buckets as it goes, and every entry is stored straight to its rank in C
//     (no sorted copy in shared memory).
// These kernels, like the hash-sort ones, are bound by the shared-memory data
// pipe (ncu on the 80^3 stencil: L1 data-pipe wavefronts 88% of peak, 32 a B
// row step, 42% of them bank conflicts), not by instruction issue or DRAM.
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"

#include <algorithm>

namespace nspb {

// Slot of `key` in a table of 2^LOG2T int slots (empty = -1), inserting it
// when absent; `fresh` tells that this call inserted it. -1 (and the error
// word) when the probe sequence is exhausted. Slots only ever change from
// empty to a key, so a stale read can only be a stale "empty", which the CAS
// corrects.
template <int LOG2T>
__device__ __forceinline__ int rg_slot(int *keys, int key, bool &fresh, int *err) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>(key);
  int cur = ((volatile int *)keys)[h];
  fresh = false;
  if (cur == key) return (int)h;
#pragma unroll 1
  for (unsigned q = 0; q <= MASK; ++q) {
    if (cur == key) return (int)h;
    if (cur == kEmpty) {
      const int old = atomicCAS(keys + h, kEmpty, key);
      if (old == kEmpty) {
        fresh = true;
        return (int)h;
      }
      if (old == key) return (int)h;
    }
    h = (h + 1u) & MASK;
    cur = ((volatile int *)keys)[h];
  }
  atomicOr(err, ERR_PROBE);
  return -1;
}

// Monotone bucket of key in [lo, lo + span): high 32 bits of (key - lo) * mul
// with mul = floor(nb * 2^32 / span), capped below 2^32 (narrow spans then
// merge neighbouring columns into one bucket, which stays monotone).
__device__ __forceinline__ unsigned rg_bucket_mul(unsigned span, int nb) {
  const unsigned long long m = ((unsigned long long)nb << 32) / (span ? span : 1u);
  return m > 0xffffffffull ? 0xffffffffu : (unsigned)m;
}
__device__ __forceinline__ int rg_bucket(int key, int lo, unsigned mul) {
  return (int)__umulhi((unsigned)key - (unsigned)lo, mul);
}

// ---- numeric ---------------------------------------------------------------------
// Per group: vals[T] (fp64, or fp32 pairs), keys[T], info[H], cnt[H], stage[G].
// After the walk the occupied slots are compacted in place to keys[0..n) with
// info = slot | (index inside the bucket << 16); the bucket-ordered keys go
// to keys[H..2H). H = the bin's largest row (T >= 2H), buckets: H.
template <int G, int LOG2H, int LOG2T>
struct NumRgCfg {
  static constexpr int T = 1 << LOG2T;
  static constexpr int H = 1 << LOG2H;
  static_assert(LOG2T > LOG2H, "table must be at least twice the row limit");
  static constexpr int V = T >= 4 * G ? 4 : (T >= 2 * G ? 2 : 1);  // slots a lane reads a round
  static constexpr int BYTES = (T * 12 + H * 8 + G * 16 + 15) & ~15;
  static constexpr int kBySmem = (56 * 1024) / BYTES > 0 ? (56 * 1024) / BYTES : 1;
  static constexpr int GPC = kBySmem < 256 / G ? kBySmem : 256 / G;
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * BYTES;
};

template <int G, int LOG2H, int LOG2T, typename VT, bool COMP, int D, bool MULTI>
__global__ void __launch_bounds__(256)
    k_num_rg(const ProdTable<VT> src, const int *__restrict__ crpt, int *__restrict__ ccol,
             double *__restrict__ cval,
             const int *__restrict__ rows, int count, int *__restrict__ err, CompArgs comp) {
  using C = NumRgCfg<G, LOG2H, LOG2T>;
  constexpr int T = C::T, H = C::H, V = C::V;
  extern __shared__ __align__(16) unsigned char smem_nrg[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  unsigned char *gb = smem_nrg + (size_t)g * C::BYTES;
  double *vals = reinterpret_cast<double *>(gb);
  float2 *vals2 = reinterpret_cast<float2 *>(gb);
  int *keys = reinterpret_cast<int *>(gb + (size_t)T * 8);
  int *info = keys + T;
  int *cnt = info + H;
  int4 *stage = reinterpret_cast<int4 *>(cnt + H);
  int *bkey = keys + H;
  int4 *k4 = reinterpret_cast<int4 *>(keys);
  int4 *c4 = reinterpret_cast<int4 *>(cnt);
  auto clear_tables = [&]() {
#pragma unroll 4
    for (int s = lane; s < T / 4; s += G) k4[s] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    for (int s = lane; s < H / 4; s += G) c4[s] = make_int4(0, 0, 0, 0);
  };
  clear_tables();
  tile.sync();

  int my_max_deg = 0, my_redo = 0;  // compensated mode, flushed once per group
  for (int r = blockIdx.x * C::GPC + g; r < count; r += gridDim.x * C::GPC) {
    const int row = rows ? rows[r] : r;
    Operands<VT> op;
    const int lr = prod_row<MULTI>(src, row, op);
    const int *acol = op.acol, *brpt = op.brpt, *bcol = op.bcol;
    const VT *aval = op.aval, *bval = op.bval;
    const int a0 = op.arpt[lr], a1 = op.arpt[lr + 1];
    const bool pair = COMP && (a1 - a0) <= comp.nmax;
    int mn = 0x7fffffff, mx = -1;
    // -- walk: one B row per step, keys of a step distinct (B rows strictly
    // increasing), so each slot has one writer per step
    for (int ab = a0; ab < a1; ab += G) {
      const int j = ab + lane;
      if (j < a1) {
        const int k = ld_stream(acol + j);
        const double av = ldv_stream(aval + j);
        const int bs = __ldg(brpt + k), be = __ldg(brpt + k + 1);
        if (be > bs) {
          mn = min(mn, __ldg(bcol + bs));
          mx = max(mx, __ldg(bcol + be - 1));
        }
        stage[lane] = make_int4(bs, be, __double2loint(av), __double2hiint(av));
      }
      tile.sync();
      const int na = min(G, a1 - ab);
      auto add = [&](int key, double a, VT b) {
        bool fresh;
        const int h = rg_slot<LOG2T>(keys, key, fresh, err);
        if (h < 0) return;
        if (pair) {
          const float af = (float)a, bf = (float)b;
          if (fresh) {
            const float ph = __fmul_rn(af, bf);
            vals2[h] = make_float2(ph, __fmaf_rn(af, bf, -ph));
          } else {
            float2 sc = vals2[h];
            comp_add(sc, af, bf);
            vals2[h] = sc;
          }
        } else {
          const double p = __dmul_rn(a, (double)b);
          vals[h] = __dadd_rn(fresh ? 0.0 : vals[h], p);
        }
      };
      int t = 0;
      if constexpr (D > 1) {
        // D B rows a round: all their keys and values are loaded before the
        // first insert; the inserts still go step by step in A-row order
        for (; t + D <= na; t += D) {
          int4 q[D];
          bool shortrows = true;
#pragma unroll
          for (int i = 0; i < D; ++i) {
            q[i] = stage[t + i];
            shortrows &= q[i].y - q[i].x <= G;
          }
          if (!shortrows) break;  // the step loop below takes the rest
          int k[D];
          VT b[D];
#pragma unroll
          for (int i = 0; i < D; ++i) {
            const int e = q[i].x + lane;
            k[i] = e < q[i].y ? __ldg(bcol + e) : -1;
            b[i] = e < q[i].y ? __ldg(bval + e) : VT(0);
          }
#pragma unroll
          for (int i = 0; i < D; ++i) {
            if (k[i] >= 0) add(k[i], __hiloint2double(q[i].w, q[i].z), b[i]);
            tile.sync();  // the next step may hit the same slots
          }
        }
      }
      for (; t < na; ++t) {
        const int4 q = stage[t];
        const double a = __hiloint2double(q.w, q.z);
        for (int e = q.x + lane; e < q.y; e += G) add(__ldg(bcol + e), a, __ldg(bval + e));
        tile.sync();  // the next step may hit the same slots
      }
    }
    mn = cg::reduce(tile, mn, cg::less<int>());
    mx = cg::reduce(tile, mx, cg::greater<int>());
    const int c0 = crpt[row];
    const int n = crpt[row + 1] - c0;
    const unsigned mul = rg_bucket_mul((unsigned)mx - (unsigned)mn + 1u, H);
    // -- compaction of the occupied slots to keys[0..n), counting buckets
    int n_occ = 0;
    for (int base = 0; base < T; base += V * G) {
      int kv[V];
      if constexpr (V == 4) {
        const int4 v = k4[base / 4 + lane];
        kv[0] = v.x; kv[1] = v.y; kv[2] = v.z; kv[3] = v.w;
      } else if constexpr (V == 2) {
        const int2 v = reinterpret_cast<const int2 *>(keys)[base / 2 + lane];
        kv[0] = v.x; kv[1] = v.y;
      } else {
        kv[0] = keys[base + lane];
      }
      int c = 0;
#pragma unroll
      for (int i = 0; i < V; ++i) c += kv[i] >= 0;
      const int incl = cg::inclusive_scan(tile, c, cg::plus<int>());
      const int tot = tile.shfl(incl, G - 1);
      tile.sync();  // every lane has read its slots before any is rewritten
      int pos = n_occ + incl - c;
#pragma unroll
      for (int i = 0; i < V; ++i) {
        if (kv[i] >= 0 && pos < H) {
          const int old = atomicAdd(&cnt[rg_bucket(kv[i], mn, mul)], 1);
          keys[pos] = kv[i];
          info[pos] = (base + V * lane + i) | (old << 16);
          ++pos;
        }
      }
      n_occ += tot;
    }
    tile.sync();
    if (n_occ != n || n > H) {  // symbolic/numeric disagreement: skip the row
      if (lane == 0) atomicOr(err, ERR_COUNT);
      clear_tables();
      tile.sync();
      continue;
    }
    // -- exclusive scan of the bucket counts (cnt becomes bucket starts)
    constexpr int PER = H >= G ? H / G : 1;
    if constexpr (PER <= 8) {  // each lane scans a run of PER counters in registers
      int local[PER];
      int sum = 0;
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int idx = lane * PER + q;
        local[q] = idx < H ? cnt[idx] : 0;
        sum += local[q];
      }
      int ex = cg::exclusive_scan(tile, sum, cg::plus<int>());
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int idx = lane * PER + q;
        if (idx < H) cnt[idx] = ex;
        ex += local[q];
      }
    } else {  // rounds of G consecutive counters
      int run = 0;
      for (int base = 0; base < H; base += G) {
        const int v = cnt[base + lane];
        const int incl = cg::inclusive_scan(tile, v, cg::plus<int>());
        cnt[base + lane] = run + incl - v;
        run += tile.shfl(incl, G - 1);
      }
    }
    tile.sync();
    // -- keys in bucket order
    for (int q = lane; q < n; q += G) {
      const int key = keys[q];
      bkey[cnt[rg_bucket(key, mn, mul)] + (info[q] >> 16)] = key;
    }
    tile.sync();
    // -- rank inside the bucket; store straight to C
    for (int q = lane; q < n; q += G) {
      const int key = keys[q];
      const int slot = info[q] & 0xffff;
      const int b = rg_bucket(key, mn, mul);
      const int st = cnt[b], en = b + 1 < H ? cnt[b + 1] : n;
      int rank = st;
      for (int u = st; u < en; ++u) rank += bkey[u] < key;
      double v;
      if (pair) {
        const float2 sc = vals2[slot];
        v = (double)sc.x + (double)sc.y;
      } else {
        v = vals[slot];
      }
      __stcs(ccol + c0 + rank, key);
      __stcs(cval + c0 + rank, v);
    }
    if (COMP) {
      if (pair) my_max_deg = max(my_max_deg, a1 - a0);
      else ++my_redo;
    }
    tile.sync();
    clear_tables();
    tile.sync();
  }
  if (COMP && lane == 0) {
    if (my_max_deg) atomicMax(comp.max_deg, my_max_deg);
    if (my_redo) atomicAdd(comp.redo, my_redo);
  }
}

template <int G, int LOG2H, int LOG2T, typename VT, bool COMP>
static cudaError_t run_num_rg(const ProdTable<VT> &t, const int *crpt, int *ccol, double *cval,
                              const int *rows, int count, int *err, CompArgs comp, int depth,
                              cudaStream_t s) {
  using C = NumRgCfg<G, LOG2H, LOG2T>;
  // four B rows loaded ahead (measured on the 128^3 stencil: 11.18 ms with
  // one, 10.26 with two, 10.06 with four)
  (void)depth;
  auto kern = t.prod_of_row ? k_num_rg<G, LOG2H, LOG2T, VT, COMP, 4, true>
                            : k_num_rg<G, LOG2H, LOG2T, VT, COMP, 4, false>;
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(t, crpt, ccol, cval, rows, count, err, comp);
  return cudaGetLastError();
}

// Numeric bin b holds rows of at most 16 << b entries (H); the table has
// 4H slots (load <= 1/4) or, with tshift = -1, 2H.
template <int G, typename VT, bool COMP>
static cudaError_t num_rg_bin(int bin, int tshift, int depth, const ProdTable<VT> &t,
                              const int *crpt, int *ccol, double *cval, const int *rows,
                              int count, int *err, CompArgs comp, cudaStream_t s) {
#define NSPB_NRG(L2H, L2T) \
  run_num_rg<G, L2H, L2T, VT, COMP>(t, crpt, ccol, cval, rows, count, err, comp, depth, s)
  const bool big = tshift >= 0;
  switch (bin) {
    case 0: return big ? NSPB_NRG(4, 6) : NSPB_NRG(4, 5);
    case 1: return big ? NSPB_NRG(5, 7) : NSPB_NRG(5, 6);
    case 2: return big ? NSPB_NRG(6, 8) : NSPB_NRG(6, 7);
    case 3: return big ? NSPB_NRG(7, 9) : NSPB_NRG(7, 8);
    case 4: return big ? NSPB_NRG(8, 10) : NSPB_NRG(8, 9);
    default: return big ? NSPB_NRG(9, 11) : NSPB_NRG(9, 10);
  }
#undef NSPB_NRG
}

cudaError_t launch_numeric_rg(int bin, int lanes, int tshift, int depth,
                              const ProdTable<double> &t, const int *crpt, int *ccol,
                              double *cval, const int *rows, int count, int *err,
                              cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  const CompArgs none{0, nullptr, nullptr};
  if (lanes == 8)
    return num_rg_bin<8, double, false>(bin, tshift, depth, t, crpt, ccol, cval, rows, count,
                                        err, none, s);
  if (lanes == 16)
    return num_rg_bin<16, double, false>(bin, tshift, depth, t, crpt, ccol, cval, rows, count,
                                         err, none, s);
  return num_rg_bin<32, double, false>(bin, tshift, depth, t, crpt, ccol, cval, rows, count, err,
                                       none, s);
}

cudaError_t launch_numeric_comp_rg(int bin, int lanes, int tshift, int depth,
                                   const ProdTable<float> &t, const int *crpt, int *ccol,
                                   double *cval, const int *rows, int count, int nmax,
                                   int *redo, int *max_deg, int *err, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  const CompArgs comp{nmax, redo, max_deg};
  if (lanes == 8)
    return num_rg_bin<8, float, true>(bin, tshift, depth, t, crpt, ccol, cval, rows, count, err,
                                      comp, s);
  if (lanes == 16)
    return num_rg_bin<16, float, true>(bin, tshift, depth, t, crpt, ccol, cval, rows, count, err,
                                       comp, s);
  return num_rg_bin<32, float, true>(bin, tshift, depth, t, crpt, ccol, cval, rows, count, err,
                                     comp, s);
}

}  // namespace nspb
