// Numeric kernels of the row-group bins that read the entry maps recorded by
// the symbolic phase (k_sym_map in symbolic.cu): rows of at most 256 entries,
// B rows strictly increasing, fp64.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu):
//   nsp_calculate_value_col_bin_mpwarp / _each_warp :1307-1494 (shared-memory
//   hash of (column, value) slots with atomic adds, then an O(nnz^2) rank sort)
//
// The symbolic phase has already probed a hash table for every intermediate
// product to count the row's distinct columns; k_sym_map also records, per
// product, the index of its column among the row's distinct columns in order
// of first appearance. The numeric walk here then adds a*b into a dense
// value array at that index: no hash table, no probe loop, no CAS, and no
// compaction of a table before the sort. The bound is still the shared-memory
// data pipe (value updates and the sort).
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"

#include <cuda_pipeline.h>

namespace nspb {

// Sort bucket of r in [0, span) for nb buckets: high 32 bits of r * mul,
// mul ~ nb * 2^32 / span (single-precision estimate), clamped to nb - 1.
// Monotone in r, so keys in lower buckets are smaller.
__device__ __forceinline__ unsigned map_bucket_mul(unsigned span, int nb) {
  const float m = (float)nb * 4294967296.0f / (float)(span ? span : 1u);
  return m >= 4294967040.0f ? 0xffffffffu : (unsigned)m;
}
__device__ __forceinline__ int map_bucket(unsigned r, unsigned mul, int nb) {
  const int b = (int)__umulhi(r, mul);
  return b < nb - 1 ? b : nb - 1;
}

// ---- numeric from entry maps ---------------------------------------------------
// Rows of at most 256 entries whose symbolic pass recorded the entry map
// (k_sym_map): every intermediate product carries the index of its column
// among the row's distinct columns in order of first appearance, so the walk
// adds a*b into vals[index] with no hash table and no probe. The walk order
// here equals the symbolic walk's (A entries in order, each B row's entries
// in order, chunks of G A entries), so the new columns of a step are exactly
// the indices at or past the count before the step; their lanes record the
// column. Quads of the map (map_quad) give each lane one 4-byte word for four
// steps; elsewhere each product has one byte. The row
// is then sorted by the bucket counting sort over [first, last column] and
// stored at its ranks.
// Per group: vals[H] fp64, keys[H], info[H] (index inside the bucket), cnt[H],
// bkey[H] (keys in bucket order), stage[G]; with PREF two buffers of G A
// entries (values, then columns) that cp.async fills for the group's next row;
// then the row template: tk/tl/tfc[G] (B row index, length and first column
// of each A entry), trel[H] (its columns in order, less its first column) and
// tinv[H] (the entry index of each rank).
//
// Row templates (run > 1): groups take their rows in runs of `run`
// consecutive launch rows and keep the last row they sorted as a template
// (its map offset, entry count, per A entry the B row index, length and first
// column, and the outcome of its sort). A row has the template's pattern, and
// so its map bytes and its sorted order, when
//  - its map offset is the template's (the symbolic pass gave both rows one
//    map only after checking that every product column is one shift of the
//    template's), or
//  - (one chunk of A entries, one product) each B row has the template's
//    length and lies in one run of shifted B rows with the template's (B row
//    shift bits), all moved by one shift; or, where the bits cannot decide,
//    its B rows' columns minus the template's all equal that shift.
// Such a row adds the products into zeroed values at their indices, with no
// column loads, no first-appearance tracking and no sort, and stores entry
// tinv[q] at rank q with column trel[q] + the row's first column. Sums run in
// the same order from the same zero, so the values are bit for bit those of
// a sorted row.
template <int G, int LOG2H, bool PREF>
struct NumMapCfg {
  static constexpr int H = 1 << LOG2H;
  static constexpr int BYTES =
      (H * 8 + H * 16 + G * 16 + (PREF ? G * 24 : 0) + G * 12 + H * 5 + 15) & ~15;
  static constexpr int kBySmem = (56 * 1024) / BYTES > 0 ? (56 * 1024) / BYTES : 1;
  static constexpr int GPC = kBySmem < 256 / G ? kBySmem : 256 / G;
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * BYTES;
};

// VT float with COMP: fp32 inputs; rows of at most comp.nmax A entries sum
// error-free fp32 pairs (TwoProduct + TwoSum) collapsed to fp64 at the end,
// the others (every row when comp.nmax is 0) sum the exact fp64 products of
// the widened inputs.
// PREF (one product): the first G A entries (columns and values) of the
// group's next row are copied into shared memory by cp.async while the
// current row is computed, so a row starts with its B-row bounds one
// dependent load away instead of two. Measured on B200 (numeric pass): 7-point
// Laplacian 128^3 (7 A entries a row) 1.47 -> 1.16 ms; 27-point stencil
// 128^3 (27 a row) 6.63 -> 7.42 ms, where the copies add to the saturated L1
// data pipe; the host takes it for A rows of at most 12 entries on average.
template <int G, int LOG2H, typename VT, bool COMP, bool MULTI, bool PREF>
__global__ void __launch_bounds__(256)
    k_num_map(const ProdTable<VT> src, const unsigned char *__restrict__ map,
              const unsigned *__restrict__ map_off, const int *__restrict__ crpt,
              int *__restrict__ ccol, double *__restrict__ cval, const int *__restrict__ rows,
              int count, int *__restrict__ err, CompArgs comp, int run,
              const unsigned *__restrict__ bshift) {
  static_assert(!(PREF && MULTI), "prefetch serves single products");
  using C = NumMapCfg<G, LOG2H, PREF>;
  constexpr int H = C::H;
  extern __shared__ __align__(16) unsigned char smem_nmap[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  unsigned char *gb = smem_nmap + (size_t)g * C::BYTES;
  double *vals = reinterpret_cast<double *>(gb);
  float2 *vals2 = reinterpret_cast<float2 *>(gb);  // the same 8 bytes as fp32 pairs
  int *keys = reinterpret_cast<int *>(gb + (size_t)H * 8);
  int *info = keys + H;
  int *cnt = info + H;
  int *bkey = cnt + H;
  int4 *stage = reinterpret_cast<int4 *>(bkey + H);
  double *avp = reinterpret_cast<double *>(stage + G);  // PREF: [2][G] A values
  int *acp = reinterpret_cast<int *>(avp + 2 * G);      // PREF: [2][G] A columns
  // the template row's A entries: B row index, length, first column
  int *tk = reinterpret_cast<int *>(gb + (size_t)H * 24 + (size_t)G * 16 + (PREF ? G * 24 : 0));
  int *tl = tk + G;
  int *tfc = tl + G;
  int *trel = tfc + G;
  unsigned char *tinv = reinterpret_cast<unsigned char *>(trel + H);
  int4 *c4 = reinterpret_cast<int4 *>(cnt);
  // the group's template: map offset and entries of the last row it sorted,
  // and the A length of the row tk/tl/tfc hold (-1: none)
  unsigned t_mo = kNoMap;
  int t_n = -1, t_na = -1;
  for (int s = lane; s < H / 4; s += G) c4[s] = make_int4(0, 0, 0, 0);
  tile.sync();

  int my_max_deg = 0, my_redo = 0;  // compensated mode, flushed once per group
  const int rstep = gridDim.x * C::GPC;  // groups in the grid
  // the group's next launch row after r: the next in its run, else the
  // first of its next run
  auto next_r = [&](int r) {
    return (r + 1) % run != 0 ? r + 1 : (r / run + rstep) * run;
  };
  // PREF: the first G A entries of the group's row rr into buffer bi
  auto prefetch = [&](int rr, int bi) {
    if constexpr (PREF) {
      if (rr < count) {
        const int rw = rows ? rows[rr] : rr;
        const int p0 = src.one.arpt[rw], p1 = src.one.arpt[rw + 1];
        if (p0 + lane < p1) {
          __pipeline_memcpy_async(acp + bi * G + lane, src.one.acol + p0 + lane, 4);
          __pipeline_memcpy_async(reinterpret_cast<VT *>(avp + bi * G) + lane,
                                  src.one.aval + p0 + lane, sizeof(VT));
        }
      }
      __pipeline_commit();
    }
  };
  int buf = 0;
  const int r0 = (blockIdx.x * C::GPC + g) * run;
  prefetch(r0, 0);
  for (int r = r0; r < count; r = next_r(r), buf ^= 1) {
    if constexpr (PREF) {
      prefetch(next_r(r), buf ^ 1);  // the buffer the previous row read
      __pipeline_wait_prior(1);      // this row's copies have landed
      tile.sync();                   // ... for every lane of the group
    }
    const int row = rows ? rows[r] : r;
    const int c0 = crpt[row];
    const int n = crpt[row + 1] - c0;
    if (n == 0) continue;  // no products (the group touched no shared state)
    const unsigned mo = map_off[row];
    if (n > H || mo == kNoMap) {
      if (lane == 0) atomicOr(err, ERR_COUNT);
      continue;
    }
    const unsigned char *mp = map + (size_t)mo * 16;
    Operands<VT> op;
    const int lr = prod_row<MULTI>(src, row, op);
    const int *acol = op.acol, *brpt = op.brpt, *bcol = op.bcol;
    const VT *aval = op.aval, *bval = op.bval;
    const int a0 = op.arpt[lr], a1 = op.arpt[lr + 1];
    const bool pair = COMP && (a1 - a0) <= comp.nmax;
    // a row of the template: no columns, no first appearances, no sort. It
    // shares the template's map, or (checked on the first chunk below) its A
    // entries' B rows are the template's moved by one shift.
    bool hit = run > 1 && !pair && mo == t_mo && n == t_n;
    int mn = 0x7fffffff, mx = -1;
    int nk = 0;   // distinct columns before the current step (uniform)
    int pos = 0;  // products walked so far (uniform)
    // one product: index ix, column c, value p. The new columns of a step
    // hold the indices from nk on; nf counts them within the step.
    bool bad = false;
    int nf = 0;
    auto add = [&](bool has, unsigned ix, int c, double a, double b) {
      if (has && ix >= (unsigned)n) {  // not an index of this row: corrupt map
        bad = true;
        has = false;
      }
      if (hit) {
        if (has) vals[ix] = __dadd_rn(vals[ix], __dmul_rn(a, b));
        return;
      }
      const bool fresh = has && (int)ix >= nk;
      nf += __popc(tile.ballot(fresh));
      if (fresh) keys[ix] = c;
      if (!has) return;
      if (pair) {  // a and b hold fp32 values: the conversions are exact
        const float af = (float)a, bf = (float)b;
        if (fresh) {
          const float ph = __fmul_rn(af, bf);
          vals2[ix] = make_float2(ph, __fmaf_rn(af, bf, -ph));
        } else {
          float2 sc = vals2[ix];
          comp_add(sc, af, bf);
          vals2[ix] = sc;
        }
      } else {
        const double p = __dmul_rn(a, b);
        vals[ix] = __dadd_rn(fresh ? 0.0 : vals[ix], p);
      }
    };
    for (int ab = a0; ab < a1; ab += G) {
      const int j = ab + lane;
      int k = 0, bs = 0, be = 0, fc = 0;
      if (j < a1) {
        double av;
        if (PREF && ab == a0) {
          k = acp[buf * G + lane];
          av = (double)reinterpret_cast<const VT *>(avp + buf * G)[lane];
        } else {
          k = ld_stream(acol + j);
          av = ldv_stream(aval + j);
        }
        bs = __ldg(brpt + k);
        be = __ldg(brpt + k + 1);
        if (be > bs) {
          fc = __ldg(bcol + bs);
          mn = min(mn, fc);
          mx = max(mx, __ldg(bcol + be - 1));
        }
        stage[lane] = make_int4(bs, be, __double2loint(av), __double2hiint(av));
      }
      if (run > 1 && ab == a0) {
        const int na0 = a1 - a0;
        if (!hit && !pair && bshift && n == t_n && na0 <= G && na0 == t_na) {
          // every B row the row reads is the template's moved by one shift d
          // (lane 0's B row gives d), so every product column moves by d
          const int d = fc - tfc[lane < na0 ? lane : 0];
          const int d0 = tile.shfl(d, 0);
          const int len = lane < na0 ? be - bs : 0;
          const bool lens = lane >= na0 || len == tl[lane];
          const bool ok =
              lens && (lane >= na0 || len == 0 || (d == d0 && same_run(bshift, k, tk[lane])));
          const bool based = tile.shfl(be - bs, 0) > 0;
          hit = based && tile.all(ok);
          if (!hit && based && tile.all(lens)) {
            // the shift bits cannot decide (the first row of a run is far from
            // the row sorted last): compare the columns themselves
            const int tbs = len > 0 ? __ldg(brpt + tk[lane]) : 0;
            bool diff = false;
            for (int t = 0; t < na0; ++t) {
              const int s0 = tile.shfl(bs, t), s1 = tile.shfl(tbs, t), ln = tile.shfl(len, t);
              for (int e = lane; e < ln; e += G)
                diff |= (unsigned)__ldg(bcol + s0 + e) - (unsigned)__ldg(bcol + s1 + e) !=
                        (unsigned)d0;
            }
            hit = !tile.any(diff);
          }
        }
        if (hit) {
          t_mo = mo;  // the same map bytes as the template's
          for (int q = lane; q < n; q += G) vals[q] = 0.0;
        } else {
          t_na = -1;  // the row that tk/tl/tfc will hold is not sorted yet
        }
        if (na0 <= G && lane < na0 && !pair) {
          tk[lane] = k;
          tl[lane] = be - bs;
          tfc[lane] = fc;
        }
      }
      tile.sync();
      const int na = min(G, a1 - ab);
      int t = 0;
      {
        // quads of the map (map_quad): four B rows a round, one 4-byte word
        // of indices per lane; indices, columns and values loaded before the
        // first add; the adds still go step by step in A-row order
        constexpr int D = 4;
        for (; t + D <= na; t += D) {
          int4 q[D];
          int len[D];
#pragma unroll
          for (int i = 0; i < D; ++i) {
            q[i] = stage[t + i];
            len[i] = q[i].y - q[i].x;
          }
          if (!map_quad<G>(len)) break;  // the step loop below takes the rest
          const int pa = (pos + 3) & ~3;
          const unsigned w = ld_stream(reinterpret_cast<const unsigned *>(mp + pa) + lane);
          pos = pa + 4 * G;
          unsigned ix[D];
          int kc[D];
          double b[D];
#pragma unroll
          for (int i = 0; i < D; ++i) {
            const int e = q[i].x + lane;
            const bool has = lane < len[i];
            ix[i] = (w >> (8 * i)) & 0xffu;
            kc[i] = has && !hit ? __ldg(bcol + e) : 0;
            b[i] = has ? ldv(bval + e) : 0.0;
          }
#pragma unroll
          for (int i = 0; i < D; ++i) {
            add(lane < len[i], ix[i], kc[i], __hiloint2double(q[i].w, q[i].z), b[i]);
            nk += nf;
            nf = 0;
            tile.sync();  // the next step may hit the same entries
          }
        }
      }
      // the rest of the chunk: one map byte per product; four B rows loaded
      // ahead while they fit the group
      for (; t + 4 <= na; t += 4) {
        int4 q[4];
        bool fit = true;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          q[i] = stage[t + i];
          fit &= q[i].y - q[i].x <= G;
        }
        if (!fit) break;
        unsigned ix[4];
        int kc[4];
        double b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int e = q[i].x + lane;
          const bool has = e < q[i].y;
          ix[i] = has ? ld_stream(mp + pos + lane) : 0u;
          kc[i] = has && !hit ? __ldg(bcol + e) : 0;
          b[i] = has ? ldv(bval + e) : 0.0;
          pos += q[i].y - q[i].x;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          add(q[i].x + lane < q[i].y, ix[i], kc[i], __hiloint2double(q[i].w, q[i].z), b[i]);
          nk += nf;
          nf = 0;
          tile.sync();  // the next step may hit the same entries
        }
      }
      for (; t < na; ++t) {
        const int4 q = stage[t];
        const double a = __hiloint2double(q.w, q.z);
        for (int eb = q.x; eb < q.y; eb += G) {  // uniform trip count across the group
          const int e = eb + lane;
          const bool has = e < q.y;
          const unsigned ix = has ? ld_stream(mp + pos + (e - q.x)) : 0u;
          const int kc = has && !hit ? __ldg(bcol + e) : 0;
          const double bv = has ? ldv(bval + e) : 0.0;
          add(has, ix, kc, a, bv);
        }
        pos += q.y - q.x;
        nk += nf;
        nf = 0;
        tile.sync();  // the next step may hit the same entries
      }
    }
    mn = cg::reduce(tile, mn, cg::less<int>());
    if (hit) {
      if (tile.any(bad)) {
        if (lane == 0) atomicOr(err, ERR_COUNT);
      } else {
        for (int q = lane; q < n; q += G) {
          __stcs(ccol + c0 + q, trel[q] + mn);
          __stcs(cval + c0 + q, vals[tinv[q]]);
        }
        if (COMP) ++my_redo;  // a row of fp64 sums (templates never hold pairs)
      }
      tile.sync();
      continue;
    }
    mx = cg::reduce(tile, mx, cg::greater<int>());
    if (tile.any(bad) || nk != n) {  // map and row pointer disagree: skip the row
      if (lane == 0) atomicOr(err, ERR_COUNT);
      tile.sync();
      continue;
    }
    const unsigned mul = map_bucket_mul((unsigned)mx - (unsigned)mn + 1u, H);
    // -- bucket counts, each key's place inside its bucket
    for (int q = lane; q < n; q += G)
      info[q] = atomicAdd(cnt + map_bucket((unsigned)(keys[q] - mn), mul, H), 1);
    tile.sync();
    // -- exclusive scan of the bucket counts (cnt becomes bucket starts)
    constexpr int PER = H >= G ? H / G : 1;
    if constexpr (PER <= 8) {
      int local[PER];
      int sum = 0;
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int i = lane * PER + q;
        local[q] = i < H ? cnt[i] : 0;
        sum += local[q];
      }
      int ex = cg::exclusive_scan(tile, sum, cg::plus<int>());
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int i = lane * PER + q;
        if (i < H) cnt[i] = ex;
        ex += local[q];
      }
    } else {
      int acc = 0;
      for (int base = 0; base < H; base += G) {
        const int v = cnt[base + lane];
        const int incl = cg::inclusive_scan(tile, v, cg::plus<int>());
        cnt[base + lane] = acc + incl - v;
        acc += tile.shfl(incl, G - 1);
      }
    }
    tile.sync();
    // -- keys in bucket order
    for (int q = lane; q < n; q += G) {
      const int key = keys[q];
      bkey[cnt[map_bucket((unsigned)(key - mn), mul, H)] + info[q]] = key;
    }
    tile.sync();
    // -- rank inside the bucket; store straight to C
    for (int q = lane; q < n; q += G) {
      const int key = keys[q];
      const int b = map_bucket((unsigned)(key - mn), mul, H);
      const int st = cnt[b], en = b + 1 < H ? cnt[b + 1] : n;
      int rank = st;
      for (int u = st; u < en; ++u) rank += bkey[u] < key;
      double v;
      if (pair) {
        const float2 sc = vals2[q];
        v = (double)sc.x + (double)sc.y;
      } else {
        v = vals[q];
      }
      __stcs(ccol + c0 + rank, key);
      __stcs(cval + c0 + rank, v);
      if (run > 1) {
        trel[rank] = key - mn;
        tinv[rank] = (unsigned char)q;
      }
    }
    // the sorted row is the template of the rows that share its map or its
    // shifted pattern
    t_mo = run > 1 && !pair ? mo : kNoMap;
    t_n = n;
    t_na = run > 1 && !pair && a1 - a0 <= G ? a1 - a0 : -1;
    if (COMP) {
      if (pair) my_max_deg = max(my_max_deg, a1 - a0);
      else ++my_redo;
    }
    tile.sync();
    for (int s = lane; s < H / 4; s += G) c4[s] = make_int4(0, 0, 0, 0);
    tile.sync();
  }
  if constexpr (PREF) __pipeline_wait_prior(0);
  if (COMP && lane == 0) {
    if (my_max_deg) atomicMax(comp.max_deg, my_max_deg);
    if (my_redo) atomicAdd(comp.redo, my_redo);
  }
}

template <int G, int LOG2H, typename VT, bool COMP, bool MULTI, bool PREF>
static cudaError_t run_num_map_k(const ProdTable<VT> &t, const unsigned char *map,
                                 const unsigned *map_off, const int *crpt, int *ccol,
                                 double *cval, const int *rows, int count, int *err,
                                 CompArgs comp, int run, const unsigned *bshift,
                                 cudaStream_t s) {
  using C = NumMapCfg<G, LOG2H, PREF>;
  auto kern = k_num_map<G, LOG2H, VT, COMP, MULTI, PREF>;
  run = template_chunk(run, count, (const void *)kern, C::THREADS, C::SMEM, C::GPC);
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM,
                                   (count + run - 1) / run, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(t, map, map_off, crpt, ccol, cval, rows, count, err,
                                         comp, run, MULTI ? nullptr : bshift);
  return cudaGetLastError();
}

template <int G, int LOG2H, typename VT, bool COMP>
static cudaError_t run_num_map(const ProdTable<VT> &t, const unsigned char *map,
                               const unsigned *map_off, const int *crpt, int *ccol,
                               double *cval, const int *rows, int count, int *err, CompArgs comp,
                               bool pref, int run, const unsigned *bshift, cudaStream_t s) {
  if (t.prod_of_row)
    return run_num_map_k<G, LOG2H, VT, COMP, true, false>(t, map, map_off, crpt, ccol, cval,
                                                          rows, count, err, comp, run, bshift, s);
  if (pref)
    return run_num_map_k<G, LOG2H, VT, COMP, false, true>(t, map, map_off, crpt, ccol, cval,
                                                          rows, count, err, comp, run, bshift, s);
  return run_num_map_k<G, LOG2H, VT, COMP, false, false>(t, map, map_off, crpt, ccol, cval, rows,
                                                         count, err, comp, run, bshift, s);
}

template <int G, typename VT, bool COMP>
static cudaError_t num_map_bin(int bin, const ProdTable<VT> &t, const unsigned char *map,
                               const unsigned *map_off, const int *crpt, int *ccol,
                               double *cval, const int *rows, int count, int *err, CompArgs comp,
                               bool pref, int run, const unsigned *bshift, cudaStream_t s) {
#define NSPB_NMAP(L2H) \
  run_num_map<G, L2H, VT, COMP>(t, map, map_off, crpt, ccol, cval, rows, count, err, comp, pref, \
                                run, bshift, s)
  switch (bin) {
    case 0: return NSPB_NMAP(4);
    case 1: return NSPB_NMAP(5);
    case 2: return NSPB_NMAP(6);
    case 3: return NSPB_NMAP(7);
    default: return NSPB_NMAP(8);
  }
#undef NSPB_NMAP
}

cudaError_t launch_numeric_map(int bin, int lanes, const ProdTable<double> &t,
                               const unsigned char *map, const unsigned *map_off,
                               const int *crpt, int *ccol, double *cval, const int *rows,
                               int count, bool prefetch_a, int run, const unsigned *bshift, int *err,
                               cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (bin >= kMapNumBins) return cudaErrorInvalidValue;
  const CompArgs none{0, nullptr, nullptr};
  if (lanes == 8)
    return num_map_bin<8, double, false>(bin, t, map, map_off, crpt, ccol, cval, rows, count,
                                         err, none, prefetch_a, run, bshift, s);
  if (lanes == 16)
    return num_map_bin<16, double, false>(bin, t, map, map_off, crpt, ccol, cval, rows, count,
                                          err, none, prefetch_a, run, bshift, s);
  return num_map_bin<32, double, false>(bin, t, map, map_off, crpt, ccol, cval, rows, count, err,
                                        none, prefetch_a, run, bshift, s);
}

cudaError_t launch_numeric_comp_map(int bin, int lanes, const ProdTable<float> &t,
                                    const unsigned char *map, const unsigned *map_off,
                                    const int *crpt, int *ccol, double *cval, const int *rows,
                                    int count, bool prefetch_a, int run, const unsigned *bshift, int nmax,
                                    int *redo,
                                    int *max_deg, int *err, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (bin >= kMapNumBins) return cudaErrorInvalidValue;
  const CompArgs comp{nmax, redo, max_deg};
  if (lanes == 8)
    return num_map_bin<8, float, true>(bin, t, map, map_off, crpt, ccol, cval, rows, count, err,
                                       comp, prefetch_a, run, bshift, s);
  if (lanes == 16)
    return num_map_bin<16, float, true>(bin, t, map, map_off, crpt, ccol, cval, rows, count, err,
                                        comp, prefetch_a, run, bshift, s);
  return num_map_bin<32, float, true>(bin, t, map, map_off, crpt, ccol, cval, rows, count, err,
                                      comp, prefetch_a, run, bshift, s);
}

}  // namespace nspb
