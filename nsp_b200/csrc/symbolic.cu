// Symbolic phase: exact number of distinct columns of each row of C.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu):
//   nsp_set_row_nz_bin_mpwarp        :477-530  (partial warp per row)
//   nsp_set_row_nz_bin_each_tb       :535-586  (block per row, warp per A entry)
//   nsp_set_row_nz_bin_each_tb_max   :863-915  (48 KB mod-hash table)
//   nsp_set_row_nz_bin_each_tb_large :755-859  + _chunk :592-750 (fail list,
//                                     column windows for the longest rows)
// Here every kernel is persistent, so one launch covers a bin whatever its
// size. Rows of up to 3072 intermediate products use row groups with hash
// tables sized to the bin; longer rows take a whole block each (handed out by
// a ticket counter as blocks free up) and count distinct columns as bits of a
// shared-memory bitmap over the row's own column span instead of a hash table
// with a fail-and-retry path.
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"

#include <algorithm>

namespace nspb {

// ---- row groups: G lanes per row, one 2^LOG2T-slot key table per group -------
template <int G, int LOG2T>
struct SymGroupCfg {
  static constexpr int T = 1 << LOG2T;
  static constexpr int kBySmem = (48 * 1024) / (4 * T) > 0 ? (48 * 1024) / (4 * T) : 1;
  static constexpr int GPC = kBySmem < 256 / G ? kBySmem : 256 / G;  // groups per CTA
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * T * 4;
};

template <int G, int LOG2T, bool MULTI>
__global__ void __launch_bounds__(256)
    k_sym_group(const ProdTable<void> src, const int *__restrict__ rows, int count,
                int *__restrict__ row_nz, int *__restrict__ err) {
  using C = SymGroupCfg<G, LOG2T>;
  extern __shared__ __align__(16) int smem_sym[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  int *table = smem_sym + g * C::T;
  for (int r = blockIdx.x * C::GPC + g; r < count; r += gridDim.x * C::GPC) {
    const int row = rows ? rows[r] : r;
    // four slots per 16-byte store (each table starts on a 16-byte boundary)
    int4 *t4 = reinterpret_cast<int4 *>(table);
#pragma unroll 4
    for (int s = lane; s < C::T / 4; s += G) t4[s] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    tile.sync();
    Operands<void> o;
    const int lr = prod_row<MULTI>(src, row, o);
    const int a0 = o.arpt[lr], a1 = o.arpt[lr + 1];
    int nz = 0;
    for (int ab = a0; ab < a1; ab += G) {
      // lanes fetch up to G A entries and their B row bounds at once
      int bs = 0, be = 0;
      if (ab + lane < a1) {
        const int k = ld_stream(o.acol + ab + lane);
        bs = __ldg(o.brpt + k);
        be = __ldg(o.brpt + k + 1);
      }
      const int cnt = min(G, a1 - ab);
      for (int t = 0; t < cnt; ++t) {
        const int s0 = tile.shfl(bs, t), s1 = tile.shfl(be, t);
        for (int e = s0 + lane; e < s1; e += G)
          nz += sym_insert<LOG2T>(table, __ldg(o.bcol + e), err);
      }
    }
    nz = cg::reduce(tile, nz, cg::plus<int>());
    if (lane == 0) row_nz[row] = nz;
    tile.sync();
  }
}

// ---- row groups that also record each product's entry index ------------------
// Same count as k_sym_group, and an entry map for the numeric phase: for
// every intermediate product, the index of its column among the row's
// distinct columns in order of first appearance (one byte). The numeric
// kernel (k_num_map) then adds every product at its index with no hash probe.
// The table holds 4-byte slots (column - row's first column) << 8 | index,
// so a probe returns the index with the key; new columns of a step take
// consecutive indices from one ballot, so the new columns of a step hold the
// indices [count before the step, count after it). A group barrier after
// every step makes its inserts visible to the next: a probe that met a stale
// empty slot for a key of an earlier step would take a second index for it.
// Indices past 255 are not recorded (such rows have more than 256 entries
// and take the hash kernels).
// Layout of a row's map (map_quad decides, identically in both kernels):
// A entries in chunks of G; in a chunk, steps (one B row each) go in quads of
// four while the next four B rows each fit the group and hold at least 3G
// products together: a quad takes 4G bytes at a 4-byte boundary, lane l's
// word holding the four steps' bytes of B entry l; from the first step that
// does not start such a quad to the end of the chunk, each product takes one
// byte in walk order. Row r of the launch writes its map at
// map + bin_off + r * stride and its 16-byte unit offset to map_off[row]; a
// row whose map outgrows stride raises MAP_OVERFLOW in *flags (the host then
// drops the map).
template <int G, int LOG2T>
__device__ __forceinline__ int sym_map_product(unsigned *table, bool has, unsigned rk, int &nk,
                                               unsigned below,
                                               const cg::thread_block_tile<G> &tile,
                                               int *err) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>((int)rk);
  int idx = 0;
  bool need = false;
  if (has) {
    // slots only go from empty to a key: a stale read is a stale empty,
    // which the CAS below corrects
    unsigned cur = table[h];
#pragma unroll 1
    for (unsigned q = 0;; ++q) {
      if ((cur >> 8) == rk) {
        idx = (int)(cur & 0xffu);
        break;
      }
      if (cur == kMapEmpty) {
        need = true;
        break;
      }
      if (q == MASK) {
        atomicOr(err, ERR_PROBE);
        break;
      }
      h = (h + 1u) & MASK;
      cur = table[h];
    }
  }
  // the new columns of the step take consecutive indices in lane order
  const unsigned nm = tile.ballot(need);
  const int mine = nk + __popc(nm & below);
  nk += __popc(nm);
  if (need) {
    idx = min(mine, 255);
    const unsigned packed = (rk << 8) | (unsigned)idx;
#pragma unroll 1
    for (unsigned q = 0;; ++q) {
      // keys of a step are distinct: a lost race was for another key
      if (atomicCAS(table + h, kMapEmpty, packed) == kMapEmpty) break;
      if (q == MASK) {
        atomicOr(err, ERR_PROBE);
        break;
      }
      h = (h + 1u) & MASK;
    }
  }
  return idx;
}

// Row templates (chunk > 1). Rows of structured grids repeat the pattern of
// their neighbours: the same A row length, the same B row lengths, and
// product columns that differ from an earlier row's by one shift. Such a row
// has the earlier row's count and, entry for entry, its map, so it needs no
// hash probe at all. Each group keeps a template: per A entry the start,
// length, index and first column of its B row, and the row's first column,
// count, map offset and B column array. It is the last row the group hashed
// whose map was recorded (and that has at most kTplA A entries), moved on to
// every later row that matched it. A row with the template's A length
// matches when
//  - (one chunk of A entries, one product) each B row has the template's
//    length and lies in one run of shifted B rows with the template's (the
//    B row shift bits below), moved by the same shift as the row's first
//    column: then every product column is the template's plus that shift; or
//  - else, its columns minus the template's, product by product, all equal
//    the difference of the first columns.
// A matching row takes the template's count and map offset and nothing is
// hashed or written. Any difference sends the row through the hash walk,
// which then makes it the template. Groups take their rows in runs of `chunk`
// consecutive launch rows so that neighbours meet. The numeric pass reads a
// matched row's map at the template's offset; the walk order, and so every
// index, is the same.
constexpr int kTplA = 64;
constexpr int kMatchRun = 4;  // B rows whose columns a match loads at once

// B row shifts: bit k of bshift is set when B row k holds as many entries as
// row k-1 and every column of row k minus its first column equals the same
// difference in row k-1 (row k is row k-1 moved by one column shift). Rows
// k' < k lie in one run of such rows when bits k'+1..k are all set, and then
// row k is row k' moved by bcol[first of k] - bcol[first of k'].
__global__ void __launch_bounds__(256)
    k_brow_shift(const int *__restrict__ brpt, const int *__restrict__ bcol, int nb,
                 unsigned *__restrict__ bits) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool same = false;
  if (k > 0 && k < nb) {
    const int s0 = __ldg(brpt + k - 1), s1 = __ldg(brpt + k), e1 = __ldg(brpt + k + 1);
    const int len = e1 - s1;
    same = len == s1 - s0;
    if (same && len > 0) {
      const int d = __ldg(bcol + s1) - __ldg(bcol + s0);
      for (int e = 1; e < len && same; ++e) same = __ldg(bcol + s1 + e) - __ldg(bcol + s0 + e) == d;
    }
  }
  const unsigned w = __ballot_sync(0xffffffffu, same);
  if ((threadIdx.x & 31) == 0 && k < nb) bits[k >> 5] = w;
}

cudaError_t launch_brow_shift(const int *brpt, const int *bcol, int nb, unsigned *bits,
                              cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  k_brow_shift<<<(nb + 255) / 256, 256, 0, s>>>(brpt, bcol, nb, bits);
  return cudaGetLastError();
}

// The scalars of a group's template (shared memory keeps them out of the
// registers the hash walk needs).
struct TplHead {
  int ok, na, mn, nk;
  unsigned mo;
  int pad;
  const int *bcol;
};

template <int G, int LOG2T>
struct SymMapCfg {
  static constexpr int T = 1 << LOG2T;
  static constexpr int BYTES = T * 4 + kTplA * 16 + 32;  // table, template B rows, TplHead
  static constexpr int GPC = SymGroupCfg<G, LOG2T>::GPC;
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * BYTES;
};

template <int G, int LOG2T, bool MULTI>
__global__ void __launch_bounds__(256, MULTI ? 4 : 5)
    k_sym_map(const ProdTable<void> src, const int *__restrict__ rows, int count,
              int *__restrict__ row_nz, int *__restrict__ err, unsigned char *__restrict__ map,
              long long bin_off, int stride, unsigned *__restrict__ map_off,
              int *__restrict__ flags, int chunk, const unsigned *__restrict__ bshift) {
  using C = SymMapCfg<G, LOG2T>;
  extern __shared__ __align__(16) unsigned smem_symm[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  const unsigned below = (1u << lane) - 1u;
  unsigned *table = smem_symm + (size_t)g * (C::BYTES / 4);
  // template, per A entry: B row start, length, B row index, first column
  int4 *tb = reinterpret_cast<int4 *>(table + C::T);
  TplHead *th = reinterpret_cast<TplHead *>(tb + kTplA);
  const bool use_tpl = chunk > 1;
  if (lane == 0) th->ok = 0;
  tile.sync();
  const int nchunks = (int)(((long long)count + chunk - 1) / chunk);
  for (int ch = blockIdx.x * C::GPC + g; ch < nchunks; ch += gridDim.x * C::GPC) {
    const int rend = (int)min((long long)count, (long long)(ch + 1) * chunk);
    for (int r = ch * chunk; r < rend; ++r) {
      const int row = rows ? rows[r] : r;
      Operands<void> o;
      const int lr = prod_row<MULTI>(src, row, o);
      const int a0 = o.arpt[lr], a1 = o.arpt[lr + 1];
      const int na = a1 - a0;
      // B row bounds of the first G A entries, and the row's first column
      int bs = 0, be = 0, mn = 0x7fffffff, k0 = 0, fc0 = 0;
      if (a0 + lane < a1) {
        k0 = ld_stream(o.acol + a0 + lane);
        bs = __ldg(o.brpt + k0);
        be = __ldg(o.brpt + k0 + 1);
        if (be > bs) mn = fc0 = __ldg(o.bcol + bs);
      }
      for (int j = a0 + G + lane; j < a1; j += G) {
        const int k = __ldg(o.acol + j);
        const int s0 = __ldg(o.brpt + k), s1 = __ldg(o.brpt + k + 1);
        if (s1 > s0) mn = min(mn, __ldg(o.bcol + s0));
      }
      mn = cg::reduce(tile, mn, cg::less<int>());
      bool hit = false;
      if (th->ok && na == th->na) {
        // every product's column minus the template's must equal this shift
        const unsigned delta = (unsigned)mn - (unsigned)th->mn;
        // one chunk of A entries whose B rows each lie in one run of shifted
        // rows with the template's, moved by delta: every product column is
        // the template's plus delta, with no column compared
        if (bshift && na <= G) {
          bool ok = true;
          if (lane < na) {
            const int4 tt = tb[lane];
            ok = be - bs == tt.y &&
                 (tt.y == 0 || ((unsigned)fc0 - (unsigned)tt.w == delta && same_run(bshift, k0, tt.z)));
          }
          hit = tile.all(ok);
        }
      }
      if (!hit && th->ok && na == th->na) {
        const unsigned delta = (unsigned)mn - (unsigned)th->mn;
        const int *t_bcol = th->bcol;
        bool bad = false;
        int mbs = bs, mbe = be;
        for (int ab = a0; ab < a1; ab += G) {
          if (ab > a0) {
            mbs = mbe = 0;
            if (ab + lane < a1) {
              const int k = ld_stream(o.acol + ab + lane);
              mbs = __ldg(o.brpt + k);
              mbe = __ldg(o.brpt + k + 1);
            }
          }
          const bool lb = ab + lane < a1 && mbe - mbs != tb[ab - a0 + lane].y;
          if (tile.any(lb)) {
            bad = true;
            break;
          }
          const int cnt = min(G, a1 - ab);
          bool cb = false;
          int t = 0;
          // first G entries of kMatchRun B rows at a time (their loads in flight
          // together), then the rest of any longer B row
          bool longer = false;
          for (; t + kMatchRun <= cnt; t += kMatchRun) {
            unsigned x[kMatchRun], y[kMatchRun];
#pragma unroll
            for (int i = 0; i < kMatchRun; ++i) {
              const int s0 = tile.shfl(mbs, t + i);
              const int4 tt = tb[ab - a0 + t + i];
              const bool h = lane < tt.y;
              longer |= tt.y > G;
              x[i] = h ? (unsigned)__ldg(o.bcol + s0 + lane) : delta;
              y[i] = h ? (unsigned)__ldg(t_bcol + tt.x + lane) : 0u;
            }
#pragma unroll
            for (int i = 0; i < kMatchRun; ++i) cb |= x[i] - y[i] != delta;
          }
          for (; t < cnt; ++t) {
            const int s0 = tile.shfl(mbs, t);
            const int4 tt = tb[ab - a0 + t];
            longer |= tt.y > G;
            if (lane < tt.y)
              cb |= (unsigned)__ldg(o.bcol + s0 + lane) - (unsigned)__ldg(t_bcol + tt.x + lane) !=
                    delta;
          }
          if (longer) {  // uniform: tb is read by every lane alike
            for (t = 0; t < cnt; ++t) {
              const int s0 = tile.shfl(mbs, t);
              const int4 tt = tb[ab - a0 + t];
              for (int e = G + lane; e < tt.y; e += G)
                cb |= (unsigned)__ldg(o.bcol + s0 + e) - (unsigned)__ldg(t_bcol + tt.x + e) !=
                      delta;
            }
          }
          if (tile.any(cb)) {
            bad = true;
            break;
          }
        }
        hit = !bad;
      }
      if (hit) {
        if (lane == 0) {
          row_nz[row] = th->nk;
          map_off[row] = th->mo;
        }
        if (bshift && na <= G) {
          // the row stands in for the template from here on (same count and
          // map): the next rows' shift check then spans a few rows, not the
          // distance back to the row that was hashed
          if (lane < na) tb[lane] = make_int4(bs, be - bs, k0, fc0);
          if (lane == 0) {
            th->mn = mn;
            th->bcol = o.bcol;
          }
          tile.sync();
        }
        continue;
      }
      // hash walk
      uint4 *t4 = reinterpret_cast<uint4 *>(table);
#pragma unroll 4
      for (int s = lane; s < C::T / 4; s += G)
        t4[s] = make_uint4(kMapEmpty, kMapEmpty, kMapEmpty, kMapEmpty);
      tile.sync();  // the table is clear, and the old template is read
      const bool rec = use_tpl && na <= kTplA;  // this row may become the template
      unsigned char *mp = map + bin_off + (size_t)r * stride;
      int nk = 0;   // distinct columns so far (uniform across the group)
      int pos = 0;  // map bytes so far, saturated at stride + 1
      for (int ab = a0; ab < a1; ab += G) {
        if (ab > a0) {
          bs = be = 0;
          if (ab + lane < a1) {
            const int k = ld_stream(o.acol + ab + lane);
            bs = __ldg(o.brpt + k);
            be = __ldg(o.brpt + k + 1);
          }
        }
        if (rec && ab + lane < a1) {
          // the first chunk keeps its B row indices and first columns (k0, fc0)
          // for the shift check; later chunks are only ever compared column by column
          tb[ab - a0 + lane] = ab == a0 ? make_int4(bs, be - bs, k0, fc0) : make_int4(bs, be - bs, 0, 0);
        }
        const int cnt = min(G, a1 - ab);
        int t = 0;
        // quads: one 4-byte word per lane
        for (; t + 4 <= cnt; t += 4) {
          int s0[4], len[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            s0[i] = tile.shfl(bs, t + i);
            len[i] = tile.shfl(be, t + i) - s0[i];
          }
          if (!map_quad<G>(len)) break;
          // the four B rows' columns are loaded before the first insert (the
          // group barrier of each step would otherwise hold the next load back)
          unsigned rks[4];
#pragma unroll
          for (int i = 0; i < 4; ++i)
            rks[i] = lane < len[i] ? (unsigned)(__ldg(o.bcol + s0[i] + lane) - mn) : 0u;
          unsigned word = 0;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const bool has = lane < len[i];
            const unsigned rk = rks[i];
            const int idx = sym_map_product<G, LOG2T>(table, has, rk, nk, below, tile, err);
            word |= (unsigned)idx << (8 * i);
            tile.sync();  // the next step sees this step's inserts
          }
          const int pa = (pos + 3) & ~3;
          if (pa + 4 * G <= stride) reinterpret_cast<unsigned *>(mp + pa)[lane] = word;
          pos = min(pa + 4 * G, stride + 1);
        }
        // the rest of the chunk: one byte per product
        for (; t < cnt; ++t) {
          const int s0 = tile.shfl(bs, t), s1 = tile.shfl(be, t);
          unsigned char *sp = mp + pos - s0;  // sp[e]: the byte of B entry e
          const int room = stride - pos;
          for (int eb = s0; eb < s1; eb += G) {  // uniform trip count across the group
            const int e = eb + lane;
            const bool has = e < s1;
            const unsigned rk = has ? (unsigned)(__ldg(o.bcol + e) - mn) : 0u;
            const int idx = sym_map_product<G, LOG2T>(table, has, rk, nk, below, tile, err);
            if (has && e - s0 < room) sp[e] = (unsigned char)idx;
          }
          pos = (int)min((long long)pos + (s1 - s0), (long long)stride + 1);
          tile.sync();  // the next step sees this step's inserts
        }
      }
      const unsigned mo =
          pos <= stride ? (unsigned)((bin_off + (long long)r * stride) >> 4) : kNoMap;
      if (lane == 0) {
        row_nz[row] = nk;
        map_off[row] = mo;
        if (mo == kNoMap) atomicOr(flags, MAP_OVERFLOW);
      }
      if (use_tpl && lane == 0) {
        th->ok = rec && mo != kNoMap;
        th->na = na;
        th->mn = mn;
        th->nk = nk;
        th->mo = mo;
        th->bcol = o.bcol;
      }
      tile.sync();
    }
  }
}

// ---- rows of more than 3072 intermediate products: one block per row ---------
// Distinct columns are counted as set bits of a shared-memory bitmap over the
// row's column span [lo, hi] (see row_span), in windows of 2^20 columns. A
// row whose span is wider than one window but whose products fit a 2^15-slot
// hash table at load <= 0.75 is counted in that table instead (same shared
// memory), so it takes one pass over its products rather than one per window.
// A block-diagonal batch of products, whose B has the columns of every
// product, thus costs each row only its own span.
constexpr int kWideThreads = 1024;
constexpr int kLongBits = 1 << 20;  // 128 KB of shared memory
constexpr int kLongWords = kLongBits / 32;
constexpr int kWideLog2T = 15;      // hash table of 2^15 ints: the same 128 KB
constexpr int kWideHashMax = 3 << (kWideLog2T - 2);

// Blocks per SM given to __launch_bounds__: a bitmap of more than 2^19 bits
// (64 KB) leaves room for one block per SM, which may then use 64 registers a
// thread; a narrower one admits two, at 32 registers (the 250k power-law
// product's first launch: 106 us at one block per SM, 72 us at two).
constexpr int kWideTwoBlockSmem = 64 * 1024;
__host__ __device__ constexpr int sym_wide_minb(int smem) {
  return smem <= kWideTwoBlockSmem ? 2 : 1;
}

template <bool MULTI, int MINB>
__global__ void __launch_bounds__(kWideThreads, MINB)
    k_sym_wide(const ProdTable<void> src, int b_sorted, const int *__restrict__ rows, int count,
               int *__restrict__ row_nz, int *__restrict__ err, int *__restrict__ ticket) {
  extern __shared__ __align__(16) unsigned bm[];
  __shared__ int red[kWideThreads / 32];
  __shared__ int s_slot;
  __shared__ RowQueue<kWideThreads> rq;
  __shared__ SpanScratch<kWideThreads> sc;
  row_queue_init(rq);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kWideThreads / 32;
  // block sum of c, valid in every thread; ends with a barrier
  auto block_sum = [&](int c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) red[warp] = c;
    __syncthreads();
    int t = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) t += red[w];
    __syncthreads();
    return t;
  };
  for (int r = next_row(ticket, count, &s_slot); r < count; r = next_row(ticket, count, &s_slot)) {
    const int row = rows ? rows[r] : r;
    Operands<void> o;
    const int lr = prod_row<MULTI>(src, row, o);
    const int *acol = o.acol, *brpt = o.brpt, *bcol = o.bcol;
    const int a0 = o.arpt[lr], a1 = o.arpt[lr + 1];
    const RowSpan sp = row_span<kWideThreads>(acol, brpt, bcol, a0, a1, b_sorted != 0, o.ncols,
                                              sc);
    int total = 0;
    if ((long long)sp.hi - sp.lo + 1 > kLongBits && sp.ip <= kWideHashMax) {
      int *table = reinterpret_cast<int *>(bm);
      for (int q = threadIdx.x; q < (1 << kWideLog2T); q += kWideThreads) table[q] = kEmpty;
      __syncthreads();
      int nz = 0;
      row_products<kWideThreads>(acol, (const double *)nullptr, brpt, bcol,
                                 (const double *)nullptr, a0, a1, rq,
                                 [&](int c, double, double) {
                                   nz += sym_insert<kWideLog2T, true>(table, c, err);
                                 });
      total = block_sum(nz);
    } else {
      for (long long w0 = sp.lo; w0 <= sp.hi; w0 += kLongBits) {
        const int wn = (int)min((long long)kLongBits, (long long)sp.hi - w0 + 1);
        const int words = (wn + 31) >> 5;
        const int base = (int)w0;
        for (int q = threadIdx.x; q < words; q += kWideThreads) bm[q] = 0u;
        __syncthreads();
        row_products<kWideThreads>(acol, (const double *)nullptr, brpt, bcol,
                                   (const double *)nullptr, a0, a1, rq,
                                   [&](int c, double, double) {
                                     const unsigned d = (unsigned)(c - base);
                                     if (d < (unsigned)wn) {
                                       const unsigned bit = 1u << (d & 31u);
                                       if (!(bm[d >> 5] & bit)) atomicOr(&bm[d >> 5], bit);
                                     }
                                   });
        __syncthreads();
        int c = 0;
        for (int q = threadIdx.x; q < words; q += kWideThreads) c += __popc(bm[q]);
        total += block_sum(c);
      }
    }
    if (threadIdx.x == 0) row_nz[row] = total;
  }
}

// ---- dispatch -------------------------------------------------------------------
template <int G, int LOG2T>
static cudaError_t run_sym_group(const ProdTable<void> &t, const int *rows, int count,
                                 int *row_nz, int *err, cudaStream_t s) {
  using C = SymGroupCfg<G, LOG2T>;
  auto kern = t.prod_of_row ? k_sym_group<G, LOG2T, true> : k_sym_group<G, LOG2T, false>;
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(t, rows, count, row_nz, err);
  return cudaGetLastError();
}

template <int G>
static cudaError_t sym_group_bin(int bin, const ProdTable<void> &t, const int *rows, int count,
                                 int *row_nz, int *err, cudaStream_t s) {
  switch (bin) {
    case 0: return run_sym_group<G, 5>(t, rows, count, row_nz, err, s);
    case 1: return run_sym_group<G, 6>(t, rows, count, row_nz, err, s);
    case 2: return run_sym_group<G, 7>(t, rows, count, row_nz, err, s);
    case 3: return run_sym_group<G, 8>(t, rows, count, row_nz, err, s);
    case 4: return run_sym_group<G, 9>(t, rows, count, row_nz, err, s);
    case 5: return run_sym_group<G, 10>(t, rows, count, row_nz, err, s);
    case 6: return run_sym_group<G, 11>(t, rows, count, row_nz, err, s);
    default: return run_sym_group<G, 12>(t, rows, count, row_nz, err, s);
  }
}

template <int G, int LOG2T>
static cudaError_t run_sym_map(const ProdTable<void> &t, const int *rows, int count,
                               int *row_nz, int *err, const MapArgs &m, cudaStream_t s) {
  using C = SymMapCfg<G, LOG2T>;
  auto kern = t.prod_of_row ? k_sym_map<G, LOG2T, true> : k_sym_map<G, LOG2T, false>;
  const int chunk = template_chunk(m.chunk, count, (const void *)kern, C::THREADS, C::SMEM,
                                   C::GPC);
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM,
                                   (count + chunk - 1) / chunk, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(t, rows, count, row_nz, err, m.map, m.bin_off, m.stride,
                                         m.map_off, m.flags, chunk, t.prod_of_row ? nullptr : m.bshift);
  return cudaGetLastError();
}

template <int G>
static cudaError_t sym_map_bin(int bin, const ProdTable<void> &t, const int *rows, int count,
                               int *row_nz, int *err, const MapArgs &m, cudaStream_t s) {
  switch (bin) {
    case 0: return run_sym_map<G, 5>(t, rows, count, row_nz, err, m, s);
    case 1: return run_sym_map<G, 6>(t, rows, count, row_nz, err, m, s);
    case 2: return run_sym_map<G, 7>(t, rows, count, row_nz, err, m, s);
    case 3: return run_sym_map<G, 8>(t, rows, count, row_nz, err, m, s);
    case 4: return run_sym_map<G, 9>(t, rows, count, row_nz, err, m, s);
    case 5: return run_sym_map<G, 10>(t, rows, count, row_nz, err, m, s);
    case 6: return run_sym_map<G, 11>(t, rows, count, row_nz, err, m, s);
    default: return run_sym_map<G, 12>(t, rows, count, row_nz, err, m, s);
  }
}

cudaError_t launch_symbolic_map(int bin, int lanes, const ProdTable<void> &t, const int *rows,
                                int count, int *row_nz, int *err, const MapArgs &m,
                                cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (bin >= kSymGroupBins) return cudaErrorInvalidValue;
  if (lanes == 8) return sym_map_bin<8>(bin, t, rows, count, row_nz, err, m, s);
  if (lanes == 16) return sym_map_bin<16>(bin, t, rows, count, row_nz, err, m, s);
  return sym_map_bin<32>(bin, t, rows, count, row_nz, err, m, s);
}

cudaError_t launch_symbolic_bin(int bin, int lanes, bool b_sorted, const ProdTable<void> &t,
                                const ProdInfo &info, const int *rows, int count, int *row_nz,
                                int *err, int *ticket, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (bin < kSymGroupBins) {
    if (lanes == 8) return sym_group_bin<8>(bin, t, rows, count, row_nz, err, s);
    if (lanes == 16) return sym_group_bin<16>(bin, t, rows, count, row_nz, err, s);
    return sym_group_bin<32>(bin, t, rows, count, row_nz, err, s);
  }
  // the bitmap covers one window of B's columns at most; the hash table needs
  // the full 128 KB, which it only uses when B has more columns than a window
  const int smem = (int)std::min<long long>(kLongWords, ((long long)info.max_ncols + 31) >> 5) * 4;
  const bool multi = t.prod_of_row != nullptr;
  auto kern = sym_wide_minb(smem) == 2 ? (multi ? k_sym_wide<true, 2> : k_sym_wide<false, 2>)
                                       : (multi ? k_sym_wide<true, 1> : k_sym_wide<false, 1>);
  const int grid = persistent_grid((const void *)kern, kWideThreads, smem, count, 1);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, kWideThreads, smem, s>>>(t, b_sorted ? 1 : 0, rows, count, row_nz, err, ticket);
  return cudaGetLastError();
}

}  // namespace nspb
