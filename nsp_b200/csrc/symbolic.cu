// Symbolic phase: exact number of distinct columns of each row of C.
//
// Reference counterparts (amavliut/nsp, nsp/src/nsp.cu):
//   nsp_set_row_nz_bin_mpwarp        :477-530  (partial warp per row)
//   nsp_set_row_nz_bin_each_tb       :535-586  (block per row, warp per A entry)
//   nsp_set_row_nz_bin_each_tb_max   :863-915  (48 KB mod-hash table)
//   nsp_set_row_nz_bin_each_tb_large :755-859  + _chunk :592-750 (fail list,
//                                     column windows for the longest rows)
// Here every kernel is a persistent grid-stride loop over its bin's rows, so
// one launch covers a bin whatever its size, tables are sized to the bin
// (up to 128 KB per block on sm_100), and the longest rows count distinct
// columns in a 2^20-bit shared-memory bitmap per column window instead of a
// hash table with a fail-and-retry path.
#include "common.cuh"
#include "internal.h"
#include "launch_util.h"

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

template <int G, int LOG2T>
__global__ void __launch_bounds__(256)
    k_sym_group(const int *__restrict__ arpt, const int *__restrict__ acol,
                const int *__restrict__ brpt, const int *__restrict__ bcol,
                const int *__restrict__ rows, int count, int *__restrict__ row_nz,
                int *__restrict__ err) {
  using C = SymGroupCfg<G, LOG2T>;
  extern __shared__ __align__(16) int smem_sym[];
  auto tile = cg::tiled_partition<G>(cg::this_thread_block());
  const int g = threadIdx.x / G;
  const int lane = tile.thread_rank();
  int *table = smem_sym + g * C::T;
  for (int r = blockIdx.x * C::GPC + g; r < count; r += gridDim.x * C::GPC) {
    const int row = rows ? rows[r] : r;
#pragma unroll 4
    for (int s = lane; s < C::T; s += G) table[s] = kEmpty;
    tile.sync();
    const int a0 = arpt[row], a1 = arpt[row + 1];
    int nz = 0;
    for (int ab = a0; ab < a1; ab += G) {
      // lanes fetch up to G A entries and their B row bounds at once
      int bs = 0, be = 0;
      if (ab + lane < a1) {
        const int k = ld_stream(acol + ab + lane);
        bs = __ldg(brpt + k);
        be = __ldg(brpt + k + 1);
      }
      const int cnt = min(G, a1 - ab);
      for (int t = 0; t < cnt; ++t) {
        const int s0 = tile.shfl(bs, t), s1 = tile.shfl(be, t);
        for (int e = s0 + lane; e < s1; e += G)
          nz += sym_insert<LOG2T>(table, __ldg(bcol + e), err);
      }
    }
    nz = cg::reduce(tile, nz, cg::plus<int>());
    if (lane == 0) row_nz[row] = nz;
    tile.sync();
  }
}

// ---- one block per row: 16 warps over the A entries, one shared table ---------
constexpr int kSymBlockThreads = 512;

template <int LOG2T>
__global__ void __launch_bounds__(kSymBlockThreads)
    k_sym_block(const int *__restrict__ arpt, const int *__restrict__ acol,
                const int *__restrict__ brpt, const int *__restrict__ bcol,
                const int *__restrict__ rows, int count, int *__restrict__ row_nz,
                int *__restrict__ err) {
  constexpr int T = 1 << LOG2T;
  extern __shared__ __align__(16) int smem_sym[];
  int *table = smem_sym;
  __shared__ int red[kSymBlockThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kSymBlockThreads / 32;
  for (int r = blockIdx.x; r < count; r += gridDim.x) {
    const int row = rows ? rows[r] : r;
    for (int s = threadIdx.x; s < T; s += kSymBlockThreads) table[s] = kEmpty;
    __syncthreads();
    const int a0 = arpt[row], a1 = arpt[row + 1];
    int nz = 0;
    for (int j = a0 + warp; j < a1; j += W) {
      const int k = ld_stream(acol + j);
      const int s0 = __ldg(brpt + k), s1 = __ldg(brpt + k + 1);
      for (int e = s0 + lane; e < s1; e += 32) nz += sym_insert<LOG2T>(table, __ldg(bcol + e), err);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nz += __shfl_xor_sync(0xffffffffu, nz, o);
    if (lane == 0) red[warp] = nz;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
#pragma unroll
      for (int w = 0; w < W; ++w) s += red[w];
      row_nz[row] = s;
    }
    __syncthreads();
  }
}

// ---- longest rows: distinct columns as bits of a 2^20-column window ----------
constexpr int kLongThreads = 1024;
constexpr int kLongBits = 1 << 20;  // 128 KB of shared memory
constexpr int kLongWords = kLongBits / 32;

__global__ void __launch_bounds__(kLongThreads)
    k_sym_long(const int *__restrict__ arpt, const int *__restrict__ acol,
               const int *__restrict__ brpt, const int *__restrict__ bcol,
               int ncols, const int *__restrict__ rows, int count,
               int *__restrict__ row_nz) {
  extern __shared__ __align__(16) unsigned bm[];
  __shared__ int red[kLongThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kLongThreads / 32;
  for (int r = blockIdx.x; r < count; r += gridDim.x) {
    const int row = rows ? rows[r] : r;
    const int a0 = arpt[row], a1 = arpt[row + 1];
    int total = 0;
    for (int c0 = 0; c0 < ncols; c0 += kLongBits) {
      for (int s = threadIdx.x; s < kLongWords; s += kLongThreads) bm[s] = 0u;
      __syncthreads();
      for (int j = a0 + warp; j < a1; j += W) {
        const int k = ld_stream(acol + j);
        const int s0 = __ldg(brpt + k), s1 = __ldg(brpt + k + 1);
        for (int e = s0 + lane; e < s1; e += 32) {
          const unsigned d = (unsigned)(__ldg(bcol + e) - c0);
          if (d < (unsigned)kLongBits) {
            const unsigned bit = 1u << (d & 31u);
            if (!(bm[d >> 5] & bit)) atomicOr(&bm[d >> 5], bit);
          }
        }
      }
      __syncthreads();
      int c = 0;
      for (int s = threadIdx.x; s < kLongWords; s += kLongThreads) c += __popc(bm[s]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) red[warp] = c;
      __syncthreads();
      if (threadIdx.x == 0)
        for (int w = 0; w < W; ++w) total += red[w];
      __syncthreads();
    }
    if (threadIdx.x == 0) row_nz[row] = total;
  }
}

// ---- dispatch -------------------------------------------------------------------
template <int G, int LOG2T>
static cudaError_t run_sym_group(const CsrDev &A, const CsrDev &B, const int *rows,
                                 int count, int *row_nz, int *err, cudaStream_t s) {
  using C = SymGroupCfg<G, LOG2T>;
  const void *f = (const void *)k_sym_group<G, LOG2T>;
  const int grid = persistent_grid(f, C::THREADS, C::SMEM, count, C::GPC);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  k_sym_group<G, LOG2T><<<grid, C::THREADS, C::SMEM, s>>>(A.rpt, A.col, B.rpt, B.col, rows,
                                                          count, row_nz, err);
  return cudaGetLastError();
}

template <int G>
static cudaError_t sym_group_bin(int bin, const CsrDev &A, const CsrDev &B, const int *rows,
                                 int count, int *row_nz, int *err, cudaStream_t s) {
  switch (bin) {
    case 0: return run_sym_group<G, 5>(A, B, rows, count, row_nz, err, s);
    case 1: return run_sym_group<G, 6>(A, B, rows, count, row_nz, err, s);
    case 2: return run_sym_group<G, 7>(A, B, rows, count, row_nz, err, s);
    case 3: return run_sym_group<G, 8>(A, B, rows, count, row_nz, err, s);
    case 4: return run_sym_group<G, 9>(A, B, rows, count, row_nz, err, s);
    case 5: return run_sym_group<G, 10>(A, B, rows, count, row_nz, err, s);
    case 6: return run_sym_group<G, 11>(A, B, rows, count, row_nz, err, s);
    default: return run_sym_group<G, 12>(A, B, rows, count, row_nz, err, s);
  }
}

template <int LOG2T>
static cudaError_t run_sym_block(const CsrDev &A, const CsrDev &B, const int *rows, int count,
                                 int *row_nz, int *err, cudaStream_t s) {
  const int smem = (1 << LOG2T) * 4;
  const void *f = (const void *)k_sym_block<LOG2T>;
  const int grid = persistent_grid(f, kSymBlockThreads, smem, count, 1);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  k_sym_block<LOG2T><<<grid, kSymBlockThreads, smem, s>>>(A.rpt, A.col, B.rpt, B.col, rows,
                                                          count, row_nz, err);
  return cudaGetLastError();
}

cudaError_t launch_symbolic_bin(int bin, int lanes, const CsrDev &A, const CsrDev &B,
                                const int *rows, int count, int *row_nz, int *err,
                                cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (bin < kSymGroupBins) {
    if (lanes == 8) return sym_group_bin<8>(bin, A, B, rows, count, row_nz, err, s);
    if (lanes == 16) return sym_group_bin<16>(bin, A, B, rows, count, row_nz, err, s);
    return sym_group_bin<32>(bin, A, B, rows, count, row_nz, err, s);
  }
  switch (bin) {
    case kSymGroupBins: return run_sym_block<13>(A, B, rows, count, row_nz, err, s);
    case kSymGroupBins + 1: return run_sym_block<14>(A, B, rows, count, row_nz, err, s);
    case kSymGroupBins + 2: return run_sym_block<15>(A, B, rows, count, row_nz, err, s);
    default: {
      const int smem = kLongWords * 4;
      const void *f = (const void *)k_sym_long;
      const int grid = persistent_grid(f, kLongThreads, smem, count, 1);
      if (grid <= 0) return cudaErrorInvalidConfiguration;
      k_sym_long<<<grid, kLongThreads, smem, s>>>(A.rpt, A.col, B.rpt, B.col, B.ncols, rows,
                                                  count, row_nz);
      return cudaGetLastError();
    }
  }
}

}  // namespace nspb
