// Row-group kernels over column chunks: a column c is the bit (c & 31) of
// the chunk c >> 5, so a row's columns are kept as a small hash table of
// (chunk id, 32-bit mask) instead of one slot per column.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu): the row-group hash
// kernels nsp_set_row_nz_bin_mpwarp / _each_tb (:477-586, symbolic) and
// nsp_calculate_value_col_bin_mpwarp / _each_warp (:1307-1494, numeric with
// the rank sort). Same results (bit-exact structure, values summed in A-row
// order), different data structure.
//
// Why chunks. The row-group hash kernels are bound by the shared-memory data
// pipe: every intermediate product probes a random slot and updates a random
// 8-byte value, at about 2-4 bank-conflicted wavefronts per warp access. In
// most sparse matrices a B row's columns come in runs (stencils, banded,
// FEM and AMG operators), so the lanes of one step fall into a few chunks:
//   - lanes of a step with the same chunk are grouped by __match_any_sync;
//     their bits are OR-ed by __reduce_or_sync and one leader per chunk
//     probes the chunk table and ORs the bits in (symbolic count = new bits);
//   - numeric, second walk: the rank of column c inside the sorted row is
//     base[chunk] + popc(mask & bits below c), so each product adds into a
//     dense accumulator at its output position; lanes of one run hit
//     consecutive addresses, and no per-row sort of columns is needed (only
//     the row's chunks, a few dozen, are ordered).
// The numeric kernel walks the products twice (chunk masks, then values);
// the host takes it when the symbolic pass found runs (columns per chunk
// well above one), and the hash kernels otherwise.
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"

#include <algorithm>

namespace nspb {

// Chunk table slot of chunk id q (>= 0), inserting it when absent; -1 and the
// error word when the table is full. Slots only go from empty to an id.
template <int LOG2T>
__device__ __forceinline__ int chunk_slot(int *cid, int q, int &fresh, int *err) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>(q);
#pragma unroll 1
  for (unsigned p = 0; p <= MASK; ++p) {
    int cur = ((volatile int *)cid)[h];
    if (cur == q) return (int)h;
    if (cur == kEmpty) {
      cur = atomicCAS(cid + h, kEmpty, q);
      if (cur == kEmpty) {
        fresh = 1;
        return (int)h;
      }
      if (cur == q) return (int)h;
    }
    h = (h + 1u) & MASK;
  }
  atomicOr(err, ERR_PROBE);
  return -1;
}

// Slot of chunk id q known to be in the table (read-only probe).
template <int LOG2T>
__device__ __forceinline__ int chunk_find(const int *cid, int q) {
  constexpr unsigned MASK = (1u << LOG2T) - 1u;
  unsigned h = hash_slot<LOG2T>(q);
#pragma unroll 1
  for (unsigned p = 0; p <= MASK; ++p) {
    const int cur = cid[h];
    if (cur == q) return (int)h;
    if (cur == kEmpty) return -1;
    h = (h + 1u) & MASK;
  }
  return -1;
}

// One step's columns into the chunk table: lanes holding a column (key >= 0)
// group by chunk; each group's leader ORs the group's bits into the chunk's
// mask. Returns the number of columns this lane's group added (leader only)
// and counts the chunks it inserted into *new_chunks. tmask: the lanes of
// this lane group (warp-level bit mask).
// GM selects how a chunk's lanes are grouped. The keys of one step are one B
// row's columns, strictly increasing across the lanes that hold them (lanes
// 0..len-1 of the group), so the lanes of a chunk are a contiguous run:
//   GM 0: runs found from the left neighbour's chunk (shfl_up); the run's bits
//         OR-ed by a segmented doubling scan of shfl_down;
//   GM 1: runs as masks from a ballot of the run heads, bits OR-ed by one
//         __reduce_or_sync over the run;
//   GM 2: __match_any_sync on the chunk id (any order of keys).
template <int LOG2T, int GM, int G>
__device__ __forceinline__ int chunk_or(int *cid, unsigned *cmask, int key, unsigned tmask,
                                        int &new_chunks, int *err) {
  const int wl = threadIdx.x & 31;
  const int gl = wl & (G - 1);  // lane inside the group
  const unsigned bit = key >= 0 ? 1u << (key & 31) : 0u;
  unsigned bits;
  bool leader;
  int q;
  if constexpr (GM == 2) {
    q = key >= 0 ? (key >> 5) : -1;
    const unsigned peers = __match_any_sync(tmask, q);
    bits = __reduce_or_sync(peers, bit);
    leader = q >= 0 && wl == __ffs(peers) - 1;
  } else {
    q = key >= 0 ? (key >> 5) : -1 - gl;  // lanes without a key: distinct, never a chunk id
    const int qp = __shfl_up_sync(tmask, q, 1, G);
    const bool head = gl == 0 || qp != q;
    leader = key >= 0 && head;
    if constexpr (GM == 0) {
      bits = bit;
#pragma unroll
      for (int d = 1; d < G; d <<= 1) {
        const unsigned t = __shfl_down_sync(tmask, bits, d, G);
        const int qn = __shfl_down_sync(tmask, q, d, G);
        if (gl + d < G && qn == q) bits |= t;
      }
    } else {
      const unsigned heads = __ballot_sync(tmask, head);
      const unsigned upto = heads & (0xffffffffu >> (31 - wl));  // heads at or below this lane
      const int first = 31 - __clz(upto);                         // this lane's run head
      const unsigned above = heads & ~(0xffffffffu >> (31 - wl)); // heads above this lane
      const unsigned gtop = tmask & ~(tmask >> 1) ? (tmask & ~(tmask >> 1)) : 0x80000000u;
      const int last = above ? __ffs(above) - 2 : 31 - __clz(gtop);
      const unsigned run = (0xffffffffu >> (31 - last)) & ~((1u << first) - 1u);
      bits = __reduce_or_sync(run, bit);
    }
  }
  if (!leader) return 0;
  int fresh = 0;
  const int s = chunk_slot<LOG2T>(cid, q, fresh, err);
  new_chunks += fresh;
  if (s < 0) return 0;
  const unsigned old = atomicOr(cmask + s, bits);
  return __popc(bits & ~old);
}

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) {
    return 0xffffffffu;
  } else {
    const unsigned base = (threadIdx.x & 31) & ~(unsigned)(G - 1);
    return ((1u << G) - 1u) << base;
  }
}

// ---- symbolic ----------------------------------------------------------------------
// Per group: cid[T] (chunk ids, -1 empty), cmask[T], stage[G]. T as the hash
// kernel of the same bin: a row of ub distinct columns has at most ub chunks.
template <int G, int LOG2T>
struct SymChunkCfg {
  static constexpr int T = 1 << LOG2T;
  static constexpr int BYTES = T * 8 + G * 8;
  static constexpr int kBySmem = (48 * 1024) / BYTES > 0 ? (48 * 1024) / BYTES : 1;
  static constexpr int GPC = kBySmem < 256 / G ? kBySmem : 256 / G;
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * BYTES;
};

template <int G, int LOG2T, int GM>
__global__ void __launch_bounds__(256)
    k_sym_chunk(const int *__restrict__ arpt, const int *__restrict__ acol,
                const int *__restrict__ brpt, const int *__restrict__ bcol,
                const int *__restrict__ rows, int count, int *__restrict__ row_nz,
                unsigned long long *__restrict__ chunks_total, int *__restrict__ err) {
  using C = SymChunkCfg<G, LOG2T>;
  constexpr int T = C::T;
  extern __shared__ __align__(16) unsigned char smem_sch[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  const unsigned tmask = group_mask<G>();
  int *cid = reinterpret_cast<int *>(smem_sch + (size_t)g * C::BYTES);
  unsigned *cmask = reinterpret_cast<unsigned *>(cid + T);
  int2 *stage = reinterpret_cast<int2 *>(cmask + T);
  auto clear = [&]() {
    int4 *c4 = reinterpret_cast<int4 *>(cid);
#pragma unroll 4
    for (int s = lane; s < T / 4; s += G) c4[s] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    int4 *m4 = reinterpret_cast<int4 *>(cmask);
#pragma unroll 4
    for (int s = lane; s < T / 4; s += G) m4[s] = make_int4(0, 0, 0, 0);
  };
  clear();
  tile.sync();
  int nch = 0;  // chunks this lane inserted (leader of its chunk group)
  for (int r = blockIdx.x * C::GPC + g; r < count; r += gridDim.x * C::GPC) {
    const int row = rows ? rows[r] : r;
    const int a0 = arpt[row], a1 = arpt[row + 1];
    int nz = 0;
    for (int ab = a0; ab < a1; ab += G) {
      const int j = ab + lane;
      if (j < a1) {
        const int k = ld_stream(acol + j);
        stage[lane] = make_int2(__ldg(brpt + k), __ldg(brpt + k + 1));
      }
      tile.sync();
      const int na = min(G, a1 - ab);
      int t = 0;
      for (; t + 2 <= na; t += 2) {  // two B rows' keys loaded before either is added
        const int2 q0 = stage[t], q1 = stage[t + 1];
        if (q0.y - q0.x <= G && q1.y - q1.x <= G) {
          const int e0 = q0.x + lane, e1 = q1.x + lane;
          const int k0 = e0 < q0.y ? __ldg(bcol + e0) : -1;
          const int k1 = e1 < q1.y ? __ldg(bcol + e1) : -1;
          nz += chunk_or<LOG2T, GM, G>(cid, cmask, k0, tmask, nch, err);
          nz += chunk_or<LOG2T, GM, G>(cid, cmask, k1, tmask, nch, err);
        } else {
          for (int i = 0; i < 2; ++i) {
            const int2 q = i ? q1 : q0;
            for (int e0 = q.x; e0 < q.y; e0 += G) {  // uniform trip count
              const int e = e0 + lane;
              nz += chunk_or<LOG2T, GM, G>(cid, cmask, e < q.y ? __ldg(bcol + e) : -1, tmask, nch, err);
            }
          }
        }
      }
      if (t < na) {
        const int2 q = stage[t];
        for (int e0 = q.x; e0 < q.y; e0 += G) {
          const int e = e0 + lane;
          nz += chunk_or<LOG2T, GM, G>(cid, cmask, e < q.y ? __ldg(bcol + e) : -1, tmask, nch, err);
        }
      }
      tile.sync();  // stage reads done before the next chunk of A entries
    }
    nz = cg::reduce(tile, nz, cg::plus<int>());
    if (lane == 0) row_nz[row] = nz;
    tile.sync();
    clear();
    tile.sync();
  }
  // chunks of every row of this group: the host's measure of column runs
  const int tot = cg::reduce(tile, nch, cg::plus<int>());
  if (chunks_total && lane == 0 && tot) atomicAdd(chunks_total, (unsigned long long)tot);
}

template <int G, int LOG2T>
static cudaError_t run_sym_chunk(const CsrDev &A, const CsrDev &B, const int *rows, int count,
                                 int *row_nz, unsigned long long *chunks, int *err, int gm,
                                 cudaStream_t s) {
  using C = SymChunkCfg<G, LOG2T>;
  auto kern = gm == 2 ? k_sym_chunk<G, LOG2T, 2>
            : gm == 1 ? k_sym_chunk<G, LOG2T, 1>
                      : k_sym_chunk<G, LOG2T, 0>;
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(A.rpt, A.col, B.rpt, B.col, rows, count, row_nz,
                                         chunks, err);
  return cudaGetLastError();
}

template <int G>
static cudaError_t sym_chunk_bin(int bin, const CsrDev &A, const CsrDev &B, const int *rows,
                                 int count, int *row_nz, unsigned long long *chunks, int *err,
                                 int gm, cudaStream_t s) {
  switch (bin) {
    case 0: return run_sym_chunk<G, 5>(A, B, rows, count, row_nz, chunks, err, gm, s);
    case 1: return run_sym_chunk<G, 6>(A, B, rows, count, row_nz, chunks, err, gm, s);
    case 2: return run_sym_chunk<G, 7>(A, B, rows, count, row_nz, chunks, err, gm, s);
    case 3: return run_sym_chunk<G, 8>(A, B, rows, count, row_nz, chunks, err, gm, s);
    case 4: return run_sym_chunk<G, 9>(A, B, rows, count, row_nz, chunks, err, gm, s);
    case 5: return run_sym_chunk<G, 10>(A, B, rows, count, row_nz, chunks, err, gm, s);
    case 6: return run_sym_chunk<G, 11>(A, B, rows, count, row_nz, chunks, err, gm, s);
    default: return run_sym_chunk<G, 12>(A, B, rows, count, row_nz, chunks, err, gm, s);
  }
}

cudaError_t launch_symbolic_chunk(int bin, int lanes, int gm, const CsrDev &A, const CsrDev &B,
                                  const int *rows, int count, int *row_nz,
                                  unsigned long long *chunks, int *err, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (lanes == 8) return sym_chunk_bin<8>(bin, A, B, rows, count, row_nz, chunks, err, gm, s);
  if (lanes == 16) return sym_chunk_bin<16>(bin, A, B, rows, count, row_nz, chunks, err, gm, s);
  return sym_chunk_bin<32>(bin, A, B, rows, count, row_nz, chunks, err, gm, s);
}

// ---- numeric -----------------------------------------------------------------------
// Per group (H = the bin's largest row, T = 2H chunk slots):
//   acc[H] fp64 (the row's values by output position), cid[T], cmask[T],
//   cbase[T] (first output position of each chunk), ord[H] (chunk ids, then
//   bucket-ordered ids), cslot[H], cnt[H] (bucket counts), stage[G].
template <int G, int LOG2H>
struct NumChunkCfg {
  static constexpr int H = 1 << LOG2H;
  static constexpr int T = 2 * H;
  static constexpr int BYTES = (H * 8 + T * 12 + H * 12 + G * 16 + 15) & ~15;
  static constexpr int kBySmem = (56 * 1024) / BYTES > 0 ? (56 * 1024) / BYTES : 1;
  static constexpr int GPC = kBySmem < 256 / G ? kBySmem : 256 / G;
  static constexpr int THREADS = GPC * G;
  static constexpr int SMEM = GPC * BYTES;
};

template <int G, int LOG2H, typename VT, int D, int GM>
__global__ void __launch_bounds__(256)
    k_num_chunk(const int *__restrict__ arpt, const int *__restrict__ acol,
                const VT *__restrict__ aval, const int *__restrict__ brpt,
                const int *__restrict__ bcol, const VT *__restrict__ bval,
                const int *__restrict__ crpt, int *__restrict__ ccol, double *__restrict__ cval,
                const int *__restrict__ rows, int count, int *__restrict__ err) {
  using C = NumChunkCfg<G, LOG2H>;
  constexpr int H = C::H, T = C::T;
  constexpr int LOG2T = LOG2H + 1;
  extern __shared__ __align__(16) unsigned char smem_nch[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  const unsigned tmask = group_mask<G>();
  unsigned char *gb = smem_nch + (size_t)g * C::BYTES;
  double *acc = reinterpret_cast<double *>(gb);
  int *cid = reinterpret_cast<int *>(acc + H);
  unsigned *cmask = reinterpret_cast<unsigned *>(cid + T);
  int *cbase = reinterpret_cast<int *>(cmask + T);
  int *ord = cbase + T;
  int *cslot = ord + H;
  int *cnt = cslot + H;
  int4 *stage = reinterpret_cast<int4 *>(cnt + H);
  auto clear = [&]() {
    int4 *c4 = reinterpret_cast<int4 *>(cid);
#pragma unroll 4
    for (int s = lane; s < T / 4; s += G) c4[s] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    int4 *m4 = reinterpret_cast<int4 *>(cmask);
#pragma unroll 4
    for (int s = lane; s < T / 4; s += G) m4[s] = make_int4(0, 0, 0, 0);
    int4 *n4 = reinterpret_cast<int4 *>(cnt);
    for (int s = lane; s < H / 4; s += G) n4[s] = make_int4(0, 0, 0, 0);
  };
  clear();
  tile.sync();
  for (int r = blockIdx.x * C::GPC + g; r < count; r += gridDim.x * C::GPC) {
    const int row = rows ? rows[r] : r;
    const int a0 = arpt[row], a1 = arpt[row + 1];
    const int c0 = crpt[row];
    const int n = crpt[row + 1] - c0;
    int mn = 0x7fffffff, mx = -1;
    // -- pass 1: chunk masks of the row (B rows strictly increasing)
    for (int ab = a0; ab < a1; ab += G) {
      const int j = ab + lane;
      if (j < a1) {
        const int k = ld_stream(acol + j);
        const int bs = __ldg(brpt + k), be = __ldg(brpt + k + 1);
        if (be > bs) {
          mn = min(mn, __ldg(bcol + bs));
          mx = max(mx, __ldg(bcol + be - 1));
        }
        stage[lane] = make_int4(bs, be, 0, 0);
      }
      tile.sync();
      const int na = min(G, a1 - ab);
      int nch = 0;
      for (int t = 0; t < na; ++t) {
        const int4 q = stage[t];
        for (int e0 = q.x; e0 < q.y; e0 += G) {
          const int e = e0 + lane;
          chunk_or<LOG2T, GM, G>(cid, cmask, e < q.y ? __ldg(bcol + e) : -1, tmask, nch, err);
        }
      }
      tile.sync();
    }
    mn = cg::reduce(tile, mn, cg::less<int>());
    mx = cg::reduce(tile, mx, cg::greater<int>());
    // -- the row's chunks: compact, order by id (bucket counting over the
    // chunk span), first output position of each chunk, columns of C
    int nc = 0;
    for (int base = 0; base < T; base += G) {
      const int id = cid[base + lane];
      const bool occ = id >= 0;
      const unsigned ball = tile.ballot(occ);
      const int pos = nc + __popc(ball & ((1u << lane) - 1u));
      if (occ && pos < H) {
        ord[pos] = id;
        cslot[pos] = base + lane;
      }
      nc += __popc(ball);
    }
    tile.sync();
    const int qlo = mn >> 5, qhi = mx >> 5;
    const unsigned mul = nc > 0 ? (unsigned)min(0xffffffffull,
                                                ((unsigned long long)H << 32) /
                                                    (unsigned long long)((unsigned)(qhi - qlo) + 1u))
                                : 0u;
    // monotone bucket of a chunk id in [qlo, qhi]; clamped so that no id can
    // address past the H counters
    auto bucket = [&](int id) {
      return min((int)__umulhi((unsigned)id - (unsigned)qlo, mul), H - 1);
    };
    int ntot = 0;
    for (int i = lane; i < nc && i < H; i += G) {
      atomicAdd(&cnt[bucket(ord[i])], 1);
      ntot += __popc(cmask[cslot[i]]);
    }
    ntot = cg::reduce(tile, ntot, cg::plus<int>());
    tile.sync();
    if (nc > H || ntot != n) {  // symbolic/numeric disagreement: skip the row
      if (lane == 0) atomicOr(err, ERR_COUNT);
      tile.sync();
      clear();
      tile.sync();
      continue;
    }
    {  // exclusive scan of the bucket counts
      int run = 0;
      for (int base = 0; base < H; base += G) {
        const int v = base + lane < H ? cnt[base + lane] : 0;
        const int incl = cg::inclusive_scan(tile, v, cg::plus<int>());
        if (base + lane < H) cnt[base + lane] = run + incl - v;
        run += tile.shfl(incl, G - 1);
      }
    }
    tile.sync();
    // rank each chunk among the ids of its bucket: the ids are scattered into
    // bucket order in acc's space, which is free until the values pass
    int *bid = reinterpret_cast<int *>(acc);  // H ints fit in H doubles
    int *bpos = bid + H;                      // per-bucket cursor copy
    for (int b = lane; b < H; b += G) bpos[b] = cnt[b];
    tile.sync();
    for (int i = lane; i < nc; i += G) {
      const int id = ord[i];
      bid[atomicAdd(&bpos[bucket(id)], 1)] = id;
    }
    tile.sync();
    // rank of each chunk, then the row's chunk popcounts in order
    for (int i = lane; i < nc; i += G) {
      const int id = ord[i];
      const int b = bucket(id);
      const int st = cnt[b], en = b + 1 < H ? cnt[b + 1] : nc;
      int rank = st;
      for (int u = st; u < en; ++u) rank += bid[u] < id;
      cbase[cslot[i]] = rank;  // rank for now; first output position below
    }
    tile.sync();
    // prefix of popcounts in chunk order: pop of rank r into bid[r]
    for (int i = lane; i < nc; i += G) {
      const int s = cslot[i];
      bid[cbase[s]] = __popc(cmask[s]);
    }
    tile.sync();
    {
      int run = 0;
      for (int base = 0; base < nc; base += G) {
        const int v = base + lane < nc ? bid[base + lane] : 0;
        const int incl = cg::inclusive_scan(tile, v, cg::plus<int>());
        if (base + lane < nc) bpos[base + lane] = run + incl - v;  // first position of rank r
        run += tile.shfl(incl, G - 1);
      }
    }
    tile.sync();
    // first output position of each chunk slot; columns of C
    for (int i = lane; i < nc; i += G) {
      const int s = cslot[i];
      const int first = bpos[cbase[s]];
      cbase[s] = first;
      unsigned m = cmask[s];
      const int colbase = ord[i] << 5;
      int p = c0 + first;
      while (m) {
        const int bit = __ffs(m) - 1;
        m &= m - 1u;
        __stcs(ccol + p++, colbase + bit);
      }
    }
    tile.sync();
    for (int i = lane; i < n; i += G) acc[i] = 0.0;  // acc's space was scratch until now
    tile.sync();
    // -- pass 2: values at their output positions, in A-row order
    for (int ab = a0; ab < a1; ab += G) {
      const int j = ab + lane;
      if (j < a1) {
        const int k = ld_stream(acol + j);
        const double av = ldv_stream(aval + j);
        stage[lane] = make_int4(__ldg(brpt + k), __ldg(brpt + k + 1), __double2loint(av),
                                __double2hiint(av));
      }
      tile.sync();
      const int na = min(G, a1 - ab);
      auto add = [&](int key, double a, VT b) {
        const int s = chunk_find<LOG2T>(cid, key >> 5);
        if (s < 0) {
          atomicOr(err, ERR_COUNT);
          return;
        }
        const int pos = cbase[s] + __popc(cmask[s] & ((1u << (key & 31)) - 1u));
        acc[pos] = __dadd_rn(acc[pos], __dmul_rn(a, (double)b));
      };
      int t = 0;
      if constexpr (D > 1) {
        for (; t + D <= na; t += D) {
          int4 q[D];
          bool shortrows = true;
#pragma unroll
          for (int i = 0; i < D; ++i) {
            q[i] = stage[t + i];
            shortrows &= q[i].y - q[i].x <= G;
          }
          if (!shortrows) break;
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
            tile.sync();  // the next step may add at the same positions
          }
        }
      }
      for (; t < na; ++t) {
        const int4 q = stage[t];
        const double a = __hiloint2double(q.w, q.z);
        for (int e = q.x + lane; e < q.y; e += G) add(__ldg(bcol + e), a, __ldg(bval + e));
        tile.sync();
      }
    }
    for (int i = lane; i < n; i += G) __stcs(cval + c0 + i, acc[i]);
    tile.sync();
    clear();
    tile.sync();
  }
}

template <int G, int LOG2H, typename VT>
static cudaError_t run_num_chunk(const CsrDev &A, const CsrDev &B, const VT *av, const VT *bv,
                                 const int *crpt, int *ccol, double *cval, const int *rows,
                                 int count, int *err, int depth, int gm, cudaStream_t s) {
  using C = NumChunkCfg<G, LOG2H>;
  auto kern = gm == 2 ? k_num_chunk<G, LOG2H, VT, 2, 2>
            : gm == 1 ? k_num_chunk<G, LOG2H, VT, 2, 1>
            : depth >= 4 ? k_num_chunk<G, LOG2H, VT, 4, 0>
            : depth >= 2 ? k_num_chunk<G, LOG2H, VT, 2, 0>
                         : k_num_chunk<G, LOG2H, VT, 1, 0>;
  const int grid = persistent_grid((const void *)kern, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(A.rpt, A.col, av, B.rpt, B.col, bv, crpt, ccol, cval,
                                         rows, count, err);
  return cudaGetLastError();
}

template <int G>
static cudaError_t num_chunk_bin(int bin, int depth, int gm, const CsrDev &A, const CsrDev &B,
                                 const int *crpt, int *ccol, double *cval, const int *rows,
                                 int count, int *err, cudaStream_t s) {
#define NSPB_NCH(L2H) \
  run_num_chunk<G, L2H, double>(A, B, A.val, B.val, crpt, ccol, cval, rows, count, err, depth, \
                                gm, s)
  switch (bin) {
    case 0: return NSPB_NCH(4);
    case 1: return NSPB_NCH(5);
    case 2: return NSPB_NCH(6);
    case 3: return NSPB_NCH(7);
    case 4: return NSPB_NCH(8);
    default: return NSPB_NCH(9);
  }
#undef NSPB_NCH
}

cudaError_t launch_numeric_chunk(int bin, int lanes, int depth, int gm, const CsrDev &A,
                                 const CsrDev &B, const int *crpt, int *ccol, double *cval,
                                 const int *rows, int count, int *err, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (lanes == 8) return num_chunk_bin<8>(bin, depth, gm, A, B, crpt, ccol, cval, rows, count, err, s);
  if (lanes == 16)
    return num_chunk_bin<16>(bin, depth, gm, A, B, crpt, ccol, cval, rows, count, err, s);
  return num_chunk_bin<32>(bin, depth, gm, A, B, crpt, ccol, cval, rows, count, err, s);
}

}  // namespace nspb
