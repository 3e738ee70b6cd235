// Host orchestration of the CSR product and the C ABI entry points.
//
// Flow of one product C = A·B on one stream (compare nsp_spgemm_kernel_hash,
// nsp/src/nsp.cu:2448-2488, which creates 11 streams, calls cudaMalloc and
// cudaFree for its scratch on every call, and synchronises the host 4-6 times):
//   1. B row-order check (skipped with opts.assume_sorted)
//   2. intermediate products per row -> symbolic bins          (host sync #1)
//   3. bin permutation (skipped when one bin holds every row)
//   4. one persistent kernel per non-empty symbolic bin
//   5. single-pass scan row_nz -> C.rowptr, numeric-bin histogram (host sync #2)
//   6. C.col / C.val allocated (unless provided)
//   7. bin permutation + one persistent kernel per non-empty numeric bin
// Scratch comes from a library-owned stream-ordered memory pool, so repeated
// calls do not call cudaMalloc for it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "internal.h"
#include "spgemm_host.h"

namespace nspb {

thread_local int g_last_cuda = 0;

const DevInfo &dev_info() {
  static std::mutex mu;
  static DevInfo infos[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lock(mu);
  DevInfo &d = infos[dev];
  if (d.device < 0) {
    cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t free_b = 0;
    if (cudaMemGetInfo(&free_b, &d.total_mem) != cudaSuccess) {
      cudaGetLastError();
      d.total_mem = 0;
    }
    d.device = dev;
  }
  return d;
}

// Library-owned stream-ordered pool per device; freed blocks stay cached.
static cudaMemPool_t scratch_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

int scratch_alloc(void **p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = scratch_pool();
  if (!pool) return NSPB_ERR_ALLOC;
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes < 256 ? 256 : bytes, pool, s);
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    return NSPB_ERR_ALLOC;
  }
  return NSPB_OK;
}

void scratch_free(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// Pinned staging for the two small device->host reads of a call.
HostStage *host_stage() {
  struct Holder {
    HostStage *p = nullptr;
    ~Holder() {
      if (p) cudaFreeHost(p);
    }
  };
  static thread_local Holder h;
  if (!h.p) {
    void *q = nullptr;
    if (cudaMallocHost(&q, sizeof(HostStage)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    h.p = static_cast<HostStage *>(q);
  }
  return h.p;
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Lanes per row group from the mean length of the B rows the products read
// and of A's rows. Measured on B200 (one call, C allocated inside): 32 lanes
// win from a mean B row of 8 entries up (random, AMG and stencil products).
// Below that, when A has enough rows to fill the GPU with smaller groups, 8
// lanes win on short A rows (7-point Laplacian 128^3, 7 entries a row: 3.38 ms
// with 8 lanes, 3.87 with 16, 5.11 with 32) and 16 on longer ones, which 8
// lanes stage in too many rounds (27-point stencil 96^3 times its smoothed
// aggregation prolongator, 27 A entries a row and B rows of 4.5: 3.53 ms with
// 16 lanes, 4.61 with 8, 4.00 with 32).
static int pick_lanes(double mean_b_row, double mean_a_row, int a_rows) {
  if (mean_b_row < 7.5 && a_rows >= 65536) return mean_a_row <= 8.0 ? 8 : 16;
  return 32;
}

// ---- a call --------------------------------------------------------------------
int Call::init(const nspb_csr_in *a, const nspb_csr_in *b, const nspb_opts *o) {
  nspb_default_opts(&opts);
  if (o) opts = *o;
  s = static_cast<cudaStream_t>(opts.stream);
  if (!a || !b) return NSPB_ERR_INVALID;
  if (a->nrows < 0 || a->ncols < 0 || b->nrows < 0 || b->ncols < 0) return NSPB_ERR_INVALID;
  if (a->ncols != b->nrows) return NSPB_ERR_INVALID;
  if (a->nnz < 0 || b->nnz < 0 || a->nnz > INT32_MAX || b->nnz > INT32_MAX) return NSPB_ERR_INVALID;
  if ((a->nrows > 0 && !a->rowptr) || (b->nrows > 0 && !b->rowptr)) return NSPB_ERR_INVALID;
  if ((a->nnz > 0 && (!a->col || !a->val)) || (b->nnz > 0 && (!b->col || !b->val)))
    return NSPB_ERR_INVALID;
  const int want = fp32_inputs(opts.precision) ? NSPB_F32 : NSPB_F64;
  if (opts.precision != NSPB_PREC_FP64 && !fp32_inputs(opts.precision)) return NSPB_ERR_INVALID;
  if ((a->nnz > 0 && a->val_type != want) || (b->nnz > 0 && b->val_type != want))
    return NSPB_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NSPB_ERR_NO_DEVICE;
  }
  auto fill = [&](CsrDev &d, const nspb_csr_in *m) {
    d.nrows = m->nrows;
    d.ncols = m->ncols;
    d.nnz = m->nnz;
    d.rpt = m->rowptr;
    d.col = m->col;
    if (m->val_type == NSPB_F32) d.val32 = static_cast<const float *>(m->val);
    else d.val = static_cast<const double *>(m->val);
  };
  fill(A, a);
  fill(B, b);
  n = A.nrows;
  t64 = ProdTable<double>{};
  t64.one = Operands<double>{A.rpt, A.col, A.val, B.rpt, B.col, B.val, B.ncols, B.nrows};
  t32 = ProdTable<float>{};
  t32.one = Operands<float>{A.rpt, A.col, A.val32, B.rpt, B.col, B.val32, B.ncols, B.nrows};
  info = ProdInfo{n, B.ncols, 1, B.nrows};
  lim = bin_limits(opts.sym_fill_pct, opts.num_fill_pct);
  a_nnz = A.nnz;
  table = false;
  ops = nullptr;
  if (opts.timing) {
    timing = true;
    for (auto &e : ev) cudaEventCreate(&e);
  }
  if (opts.group_lanes == 8 || opts.group_lanes == 16 || opts.group_lanes == 32) {
    lanes = opts.group_lanes;
  } else {
    // until the intermediate products are counted (symbolic): B's mean row
    const double avg = B.nrows > 0 ? (double)B.nnz / (double)B.nrows : 0.0;
    lanes = pick_lanes(avg, A.nrows > 0 ? (double)A.nnz / (double)A.nrows : 0.0, A.nrows);
  }
  return NSPB_OK;
}

void Call::set_table(const ProdTable<double> &d, const ProdTable<float> &f, const ProdInfo &pi,
                     int64_t total_a_nnz) {
  t64 = d;
  t32 = f;
  info = pi;
  n = pi.n;
  a_nnz = total_a_nnz;
  table = true;
  ops = reinterpret_cast<const Operands<void> *>(d.ops);
  A = CsrDev{};
  B = CsrDev{};
  A.nrows = pi.n;
  A.nnz = total_a_nnz;
  B.ncols = pi.max_ncols;
  if (!(opts.group_lanes == 8 || opts.group_lanes == 16 || opts.group_lanes == 32)) lanes = 32;
}

size_t Call::scratch_bytes() {
  const size_t nn = (size_t)std::max(n, 1);
  off_row_nz = 0;
  off_perm = align256(off_row_nz + (nn + 1) * 4);
  off_counters = align256(off_perm + nn * 4);
  off_tiles = align256(off_counters + sizeof(DevCounters));
  const size_t tiles = (size_t)scan_tiles(n);
  ws_bytes = align256(off_tiles + tiles * 8);
  return ws_bytes;
}

int Call::alloc_scratch() {
  scratch_bytes();
  if (ext_ws) {
    if (ws_bytes > ext_bytes) return NSPB_ERR_CAPACITY;
    ws = ext_ws;
    ws_external = true;
  } else {
    int st = scratch_alloc(reinterpret_cast<void **>(&ws), ws_bytes, s);
    if (st) return st;
  }
  row_nz = reinterpret_cast<int *>(ws + off_row_nz);
  perm = reinterpret_cast<int *>(ws + off_perm);
  ctr = reinterpret_cast<DevCounters *>(ws + off_counters);
  tile_state = reinterpret_cast<unsigned long long *>(ws + off_tiles);
  // counters and scan tile states are contiguous: one memset clears both
  cudaError_t e = cudaMemsetAsync(ws + off_counters, 0, ws_bytes - off_counters, s);
  if (e != cudaSuccess) return cuda_fail(e);
  return NSPB_OK;
}

Call::~Call() {
  if (ws && !ws_external) scratch_free(ws, s);
  if (map_block) scratch_free(map_block, s);
  for (auto &e : ev)
    if (e) cudaEventDestroy(e);
}

int Call::cuda_fail(cudaError_t e) {
  g_last_cuda = (int)e;
  cudaGetLastError();
  return NSPB_ERR_CUDA;
}

cudaError_t Call::order_block_bins(const int *key, int kind, const int *counts, int first,
                                   int end, const BinOffsets &off) {
  RowLists lists{};
  for (int b = first; b < end; ++b)
    if (counts[b] > 1) {
      lists.off[lists.n] = off.v[b];
      lists.count[lists.n] = counts[b];
      ++lists.n;
    }
  if (lists.n == 0) return cudaSuccess;
  ++launches;
  return launch_order_rows(key, kind, lists, perm, s);
}

int Call::fetch_counters() {
  HostStage *hs = stage ? stage : host_stage();
  if (!hs) return NSPB_ERR_ALLOC;
  cudaError_t e = cudaMemcpyAsync(&hs->c, ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(e);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e);
  h = hs->c;
  if (h.err) return NSPB_ERR_DEVICE;
  return NSPB_OK;
}

static BinOffsets offsets_of(const int *counts, int nb, int *nonempty, int *total) {
  BinOffsets o;
  int acc = 0, ne = 0;
  for (int b = 0; b < 16; ++b) {
    o.v[b] = acc;
    if (b < nb) {
      acc += counts[b];
      ne += counts[b] > 0;
    }
  }
  *nonempty = ne;
  *total = acc;
  return o;
}

// Steps 1-5: C.rowptr and nnz(C). crpt must hold n+1 ints.
int Call::symbolic(int *crpt, int64_t *nnz_out) {
  cudaError_t e;
  if (n == 0) {
    e = cudaMemsetAsync(crpt, 0, sizeof(int), s);
    if (e != cudaSuccess) return cuda_fail(e);
    *nnz_out = 0;
    return NSPB_OK;
  }
  int st = alloc_scratch();
  if (st) return st;
  mark(0);
  // B = A (the same arrays): the row walk of k_rowinfo checks B's order too
  const bool same = !table && A.rpt == B.rpt && A.col == B.col && A.nrows == B.nrows &&
                    A.nnz == B.nnz;
  if (!opts.assume_sorted && !same) {
    e = table ? launch_check_sorted_table(ops, info.nprod, info.max_brows, &ctr->flags, s)
              : launch_check_sorted(B, &ctr->flags, s);
    if (e != cudaSuccess) return cuda_fail(e);
    ++launches;
  }
  // perm is free until the bins are permuted: it holds the long-row list here
  if ((e = launch_rowinfo(structure_of(t64), n, a_nnz, lim, row_nz, nullptr, ctr->sym_counts,
                          &ctr->total_ip,
                          !opts.assume_sorted && same ? &ctr->flags : nullptr, perm,
                          &ctr->long_rows, s)) != cudaSuccess)
    return cuda_fail(e);
  ++launches;
  mark(1);
  if ((st = fetch_counters())) return st;
  b_sorted = opts.assume_sorted || !(h.flags & B_UNSORTED);
  intprod = (int64_t)h.total_ip;
  // the mean length of the B rows actually read, weighted by how often A reads
  // them: a block-diagonal batch mixes products whose B rows differ
  if (!(opts.group_lanes == 8 || opts.group_lanes == 16 || opts.group_lanes == 32) && a_nnz > 0)
    lanes = pick_lanes((double)intprod / (double)a_nnz, (double)a_nnz / (double)n, n);
  int nonempty = 0, binned = 0;
  BinOffsets off = offsets_of(h.sym_counts, kSymBins, &nonempty, &binned);
  const bool direct = nonempty == 1 && binned == n;
  // entry maps: a stride of the bin's row limit (products) per row
  long long map_bin_off[kSymGroupBins] = {};
  int map_stride[kSymGroupBins] = {};
  use_map = false;
  if (map_wanted()) {
    long long total = 0;
    for (int b = 0; b < kSymGroupBins; ++b) {
      // quads of the map take at most 4/3 of a byte per product, plus alignment
      map_stride[b] = (int)(((long long)lim.sym[b] * 3 / 2 + 16 + 15) & ~15LL);
      map_bin_off[b] = total;
      total += (long long)h.sym_counts[b] * map_stride[b];
    }
    const size_t head = align256((size_t)n * 4);
    // row templates of one product check B rows by their shift bits
    const bool shift_bits = !(opts.row_kernel & kNoRowTemplates) && !table;
    const size_t bits = shift_bits ? align256(((size_t)B.nrows / 32 + 1) * 4) : 0;
    // at most an eighth of the device's memory (C is allocated after this phase)
    if ((head + bits + (size_t)total) * 8 <= dev_info().total_mem &&
        scratch_alloc(&map_block, head + bits + (size_t)total, s) == NSPB_OK) {
      map_off = static_cast<unsigned *>(map_block);
      bshift = shift_bits ? reinterpret_cast<unsigned *>(static_cast<unsigned char *>(map_block) +
                                                         head)
                          : nullptr;
      map = static_cast<unsigned char *>(map_block) + head + bits;
      use_map = true;
      if (bshift) {
        if ((e = launch_brow_shift(B.rpt, B.col, B.nrows, bshift, s)) != cudaSuccess)
          return cuda_fail(e);
        ++launches;
      }
    }
  }
  mark(2);
  if (!direct && binned > 0) {
    if ((e = launch_perm(row_nz, n, 0, off, lim, ctr->cursor_sym, perm, s)) != cudaSuccess)
      return cuda_fail(e);
    ++launches;
    if ((e = order_block_bins(row_nz, 0, h.sym_counts, kSymGroupBins, kSymBins, off)) != cudaSuccess)
      return cuda_fail(e);
  }
  for (int b = 0; b < kSymBins; ++b) {
    const int c = h.sym_counts[b];
    if (c <= 0) continue;
    const int *rows = direct ? nullptr : perm + off.v[b];
    if (use_map) {
      MapArgs m;
      m.map = map;
      m.bin_off = map_bin_off[b];
      m.stride = map_stride[b];
      m.map_off = map_off;
      m.flags = &ctr->flags;
      m.chunk = template_run();
      m.bshift = bshift;
      e = launch_symbolic_map(b, lanes, structure_of(t64), rows, c, row_nz, &ctr->err, m, s);
    } else {
      e = launch_symbolic_bin(b, lanes, b_sorted, structure_of(t64), info, rows, c, row_nz,
                              &ctr->err, &ctr->ticket[b], s);
    }
    if (e != cudaSuccess) return cuda_fail(e);
    ++launches;
  }
  mark(3);
  if ((e = launch_scan(row_nz, n, crpt, &ctr->total_nnz, tile_state, &ctr->tile_ctr, lim,
                       ctr->num_counts, &ctr->err, s)) != cudaSuccess)
    return cuda_fail(e);
  ++launches;
  mark(4);
  if ((st = fetch_counters())) return st;
  num_counts_ready = true;
  if (use_map && (h.flags & MAP_OVERFLOW)) {  // a row outgrew its stride: no map
    use_map = false;
    scratch_free(map_block, s);
    map_block = nullptr;
    map = nullptr;
    map_off = nullptr;
    bshift = nullptr;
  }
  if (h.total_nnz > INT32_MAX) return NSPB_ERR_OVERFLOW;
  *nnz_out = h.total_nnz;
  return NSPB_OK;
}

// Step 7 (the numeric-bin histogram must be in h.num_counts).
int Call::numeric(const int *crpt, int *ccol, double *cval) {
  cudaError_t e;
  if (n == 0) return NSPB_OK;
  int nonempty = 0, binned = 0;
  BinOffsets off = offsets_of(h.num_counts, kNumBins, &nonempty, &binned);
  if (binned == 0) return NSPB_OK;
  const bool direct = nonempty == 1 && binned == n;
  mark(5);
  if (!direct) {
    if ((e = launch_perm(crpt, n, 1, off, lim, ctr->cursor_num, perm, s)) != cudaSuccess)
      return cuda_fail(e);
    ++launches;
    if ((e = order_block_bins(crpt, 1, h.num_counts, kNumGroupBins, kNumBins, off)) != cudaSuccess)
      return cuda_fail(e);
  }
  // fp32 inputs: rows of at most nmax A entries accumulate in fp32 pairs, the
  // others (every row in the wide mode) in fp64 from exact products
  const bool comp = fp32_inputs(opts.precision);
  const int nmax = opts.precision == NSPB_PREC_FP32_COMP ? comp_nmax(opts.comp_tol) : 0;
  const bool staged = use_staged();
  for (int b = 0; b < kNumBins; ++b) {
    const int c = h.num_counts[b];
    if (c <= 0) continue;
    const int *rows = direct ? nullptr : perm + off.v[b];
    int *ticket = &ctr->ticket[16 + b];
    const int tshift = opts.num_table_shift == 1 ? 1 : 0;
    if (use_map && b < kMapNumBins) {
      // cp.async of the next row's A entries pays on short A rows (7-point
      // Laplacian 128^3: numeric 1.47 -> 1.16 ms) and costs on long ones
      // (27-point stencil 128^3: 6.63 -> 7.42 ms, L1 data pipe saturated)
      const bool pref = !table && a_nnz <= 12LL * n;
      const int run = template_run();
      e = comp ? launch_numeric_comp_map(b, lanes, t32, map, map_off, crpt, ccol, cval, rows, c,
                                         pref, run, bshift, nmax, &ctr->redo_count,
                                         &ctr->max_comp_deg, &ctr->err, s)
               : launch_numeric_map(b, lanes, t64, map, map_off, crpt, ccol, cval, rows, c, pref,
                                    run, bshift, &ctr->err, s);
      if (e != cudaSuccess) return cuda_fail(e);
      ++launches;
      continue;
    }
    if (b < kNumGroupBins && b_sorted && staged) {
      const int rg_shift = (opts.row_kernel & 0xff) == 3 ? -1 : 0;  // tables 2x, else 4x
      e = comp ? launch_numeric_comp_rg(b, lanes, rg_shift, rg_depth(), t32, crpt, ccol, cval,
                                        rows, c, nmax, &ctr->redo_count, &ctr->max_comp_deg,
                                        &ctr->err, s)
               : launch_numeric_rg(b, lanes, rg_shift, rg_depth(), t64, crpt, ccol, cval, rows,
                                   c, &ctr->err, s);
      if (e != cudaSuccess) return cuda_fail(e);
      ++launches;
      continue;
    }
    e = comp ? launch_numeric_comp_bin(b, lanes, b_sorted, b_sorted, t32, info, crpt, ccol, cval,
                                       rows,
                                       c, nmax, &ctr->redo_count, &ctr->max_comp_deg, &ctr->err,
                                       ticket, tshift, s)
             : launch_numeric_bin(b, lanes, b_sorted, b_sorted, t64, info, crpt, ccol, cval,
                                  rows, c,
                                  &ctr->err, ticket, tshift, s);
    if (e != cudaSuccess) return cuda_fail(e);
    ++launches;
  }
  mark(6);
  return NSPB_OK;
}

// The symbolic phase records entry maps when the numeric phase of the same
// call can use them: B rows strictly increasing, every row with
// products in a row-group symbolic bin, column offsets within 24 bits, and
// row_kernel 7 (maps), or 0 (automatic) when the B rows the products read
// fill at least 3/4 of a row group's lanes on average. The map costs the
// symbolic pass a fixed amount per B row and saves the numeric pass a hash
// probe per product. Measured on B200 (full product, maps vs staged walk):
// 27-point stencil 128^3 12.9 vs 14.3 ms and 96^3 5.3 vs 5.9 ms (B rows of
// 27 on 32 lanes), 7-point Laplacian 128^3 2.13 vs 2.28 ms (7 on 8 lanes);
// slower on smoothed-aggregation products, 3.3 vs 2.5 ms for A*P of the
// 96^3 stencil (4.5 on 16 lanes), and on random products of 4..32 entries
// a row, 3.2 vs 3.0 ms (18 on 32 lanes, against the hash-sort kernels).
bool Call::map_wanted() const {
  const int k = opts.row_kernel & 0xff;
  if (!allow_map || !(k == 0 || k == 7)) return false;
  if (!b_sorted || n <= 0 || a_nnz <= 0) return false;
  if (info.max_ncols > kMapMaxCols) return false;
  for (int b = kSymGroupBins; b < kSymBins; ++b)
    if (h.sym_counts[b] > 0) return false;
  if (k == 7) return true;
  return (double)intprod >= 0.75 * (double)lanes * (double)a_nnz;
}

// Numeric bins and B order for a two-call numeric step.
int Call::prepare_numeric(const int *crpt) {
  if (n == 0) return NSPB_OK;
  int st = alloc_scratch();
  if (st) return st;
  cudaError_t e;
  if (!opts.assume_sorted) {
    e = table ? launch_check_sorted_table(ops, info.nprod, info.max_brows, &ctr->flags, s)
              : launch_check_sorted(B, &ctr->flags, s);
    if (e != cudaSuccess) return cuda_fail(e);
  }
  if ((e = launch_num_hist(crpt, n, lim, ctr->num_counts, s)) != cudaSuccess) return cuda_fail(e);
  launches += opts.assume_sorted ? 1 : 2;
  if ((st = fetch_counters())) return st;
  b_sorted = opts.assume_sorted || !(h.flags & B_UNSORTED);
  num_counts_ready = true;
  return NSPB_OK;
}

// Largest A-row degree n whose Dot2 error bound gamma_n^2 (gamma_n =
// n u / (1 - n u), u = 2^-24, Ogita, Rump and Oishi 2005) stays within tol,
// relative to sum |a_ik b_kj|; fp32 pairs then add within tol of the exact sum.
int comp_nmax(double tol) {
  if (!(tol > 0.0)) tol = 1e-10;
  const double u = 0x1.0p-24, r = std::sqrt(tol);
  return (int)std::floor(r / (u * (1.0 + r)));
}

double comp_bound(int n) {
  if (n <= 0) return 0.0;
  const double u = 0x1.0p-24, g = n * u / (1.0 - n * u);
  return g * g + 0x1.0p-53;
}

int Call::finish(nspb_stats *stats) {
  if ((opts.check_errors || opts.precision == NSPB_PREC_FP32_COMP) && n > 0) {
    int st = fetch_counters();
    if (st) return st;
  }
  if (stats) {
    stats->intprod = intprod;
    stats->nnz = h.total_nnz;
    for (int b = 0; b < 16; ++b) {
      stats->sym_bins[b] = b < kSymBins ? h.sym_counts[b] : 0;
      stats->num_bins[b] = b < kNumBins ? h.num_counts[b] : 0;
    }
    stats->b_sorted = b_sorted ? 1 : 0;
    stats->rows_redone = opts.precision == NSPB_PREC_FP32_COMP ? h.redo_count : 0;
    stats->max_row_err = opts.precision == NSPB_PREC_FP32_COMP ? comp_bound(h.max_comp_deg) : 0.0;
    stats->launches = launches;
    stats->entry_map = use_map ? 1 : 0;
    stats->ms_rowinfo = stats->ms_symbolic = stats->ms_scan = stats->ms_numeric = 0.f;
    if (timing && n > 0) {
      cudaStreamSynchronize(s);
      auto span = [&](int a, int b) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev[a], ev[b]) != cudaSuccess) {
          cudaGetLastError();
          ms = 0.f;
        }
        return ms;
      };
      stats->ms_rowinfo = span(0, 1);
      stats->ms_symbolic = span(2, 3);
      stats->ms_scan = span(3, 4);
      stats->ms_numeric = span(5, 6);
    }
  }
  return NSPB_OK;
}

int alloc_out(void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes < 4 ? 4 : bytes);
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    return NSPB_ERR_ALLOC;
  }
  return NSPB_OK;
}

}  // namespace nspb

using namespace nspb;

extern "C" {

const char *nspb_version(void) { return "nspb 0.1 (sm_100a)"; }

const char *nspb_strerror(int status) {
  switch (status) {
    case NSPB_OK: return "success";
    case NSPB_ERR_INVALID: return "invalid argument";
    case NSPB_ERR_OVERFLOW: return "nnz(C) or a row count exceeds int32";
    case NSPB_ERR_ALLOC: return "allocation failed";
    case NSPB_ERR_CUDA: return "CUDA runtime error";
    case NSPB_ERR_DEVICE: return "device error word set (bounded probe or wait exhausted)";
    case NSPB_ERR_NO_DEVICE: return "no CUDA device";
    case NSPB_ERR_UNSUPPORTED: return "unsupported";
    case NSPB_ERR_CAPACITY: return "output capacity too small";
    case NSPB_ERR_IO: return "file could not be opened, read or written";
    default: return "unknown status";
  }
}

int nspb_last_cuda_error(void) { return g_last_cuda; }

void nspb_default_opts(nspb_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = NSPB_PREC_FP64;
  o->comp_tol = 1e-10;
}

int nspb_free(void *p) {
  if (!p) return NSPB_OK;
  cudaError_t e = cudaFree(p);
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    return NSPB_ERR_CUDA;
  }
  return NSPB_OK;
}

int nspb_device_sm_count(int *sms) {
  int ndev = 0;
  if (!sms) return NSPB_ERR_INVALID;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NSPB_ERR_NO_DEVICE;
  }
  *sms = dev_info().sms;
  return NSPB_OK;
}

int nspb_spgemm_symbolic(const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                         const nspb_opts *opts, nspb_stats *stats) {
  if (!C) return NSPB_ERR_INVALID;
  Call call;
  int st = call.init(A, B, opts);
  if (st) return st;
  call.allow_map = false;  // the numeric phase runs in another call
  bool own_rpt = false;
  if (!C->rowptr) {
    if ((st = alloc_out(reinterpret_cast<void **>(&C->rowptr), ((size_t)call.n + 1) * 4))) return st;
    own_rpt = true;
  }
  int64_t nnz = 0;
  st = call.symbolic(C->rowptr, &nnz);
  if (!st) st = call.finish(stats);
  if (st) {
    if (own_rpt) {
      cudaStreamSynchronize(call.s);
      cudaFree(C->rowptr);
      C->rowptr = nullptr;
    }
    return st;
  }
  C->nrows = A->nrows;
  C->ncols = B->ncols;
  C->nnz = nnz;
  return NSPB_OK;
}

int nspb_spgemm_numeric(const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                        const nspb_opts *opts, nspb_stats *stats) {
  if (!C || !C->rowptr) return NSPB_ERR_INVALID;
  Call call;
  int st = call.init(A, B, opts);
  if (st) return st;
  if (C->nnz < 0 || C->nnz > INT32_MAX) return NSPB_ERR_INVALID;
  if ((C->col || C->val) && (!C->col || !C->val)) return NSPB_ERR_INVALID;
  if (C->col && C->capacity < C->nnz) return NSPB_ERR_CAPACITY;
  if ((st = call.prepare_numeric(C->rowptr))) return st;
  call.h.total_nnz = C->nnz;
  bool own = false;
  if (!C->col) {
    if ((st = alloc_out(reinterpret_cast<void **>(&C->col), (size_t)C->nnz * 4))) return st;
    if ((st = alloc_out(reinterpret_cast<void **>(&C->val), (size_t)C->nnz * 8))) {
      cudaFree(C->col);
      C->col = nullptr;
      return st;
    }
    own = true;
    C->capacity = C->nnz;
  }
  st = call.numeric(C->rowptr, C->col, C->val);
  if (!st) st = call.finish(stats);
  if (st && own) {
    cudaStreamSynchronize(call.s);
    cudaFree(C->col);
    cudaFree(C->val);
    C->col = nullptr;
    C->val = nullptr;
  }
  return st;
}

int nspb_spgemm(const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                const nspb_opts *opts, nspb_stats *stats) {
  if (!C) return NSPB_ERR_INVALID;
  if ((C->col || C->val) && (!C->col || !C->val)) return NSPB_ERR_INVALID;
  Call call;
  int st = call.init(A, B, opts);
  if (st) return st;
  bool own_rpt = false, own_cv = false;
  if (!C->rowptr) {
    if ((st = alloc_out(reinterpret_cast<void **>(&C->rowptr), ((size_t)call.n + 1) * 4))) return st;
    own_rpt = true;
  }
  int64_t nnz = 0;
  st = call.symbolic(C->rowptr, &nnz);
  if (!st) {
    if (!C->col) {
      st = alloc_out(reinterpret_cast<void **>(&C->col), (size_t)nnz * 4);
      if (!st) {
        st = alloc_out(reinterpret_cast<void **>(&C->val), (size_t)nnz * 8);
        if (st) {
          cudaFree(C->col);
          C->col = nullptr;
        }
      }
      own_cv = !st;
      if (!st) C->capacity = nnz;
    } else if (C->capacity < nnz) {
      st = NSPB_ERR_CAPACITY;
    }
  }
  if (!st) st = call.numeric(C->rowptr, C->col, C->val);
  if (!st) st = call.finish(stats);
  if (st) {
    cudaStreamSynchronize(call.s);
    if (own_cv) {
      cudaFree(C->col);
      cudaFree(C->val);
      C->col = nullptr;
      C->val = nullptr;
    }
    if (own_rpt) {
      cudaFree(C->rowptr);
      C->rowptr = nullptr;
    }
    return st;
  }
  C->nrows = A->nrows;
  C->ncols = B->ncols;
  C->nnz = nnz;
  return NSPB_OK;
}

int nspb_intprod(const nspb_csr_in *A, const nspb_csr_in *B, int64_t *d_row_ip, int64_t *total,
                 void *stream) {
  nspb_opts o;
  nspb_default_opts(&o);
  o.stream = stream;
  o.assume_sorted = 1;
  // values are not read: accept either value type
  o.precision = (A && A->val_type == NSPB_F32) ? NSPB_PREC_FP32_COMP : NSPB_PREC_FP64;
  Call call;
  int st = call.init(A, B, &o);
  if (st) return st;
  if (call.n == 0) {
    if (total) *total = 0;
    return NSPB_OK;
  }
  if ((st = call.alloc_scratch())) return st;
  cudaError_t e = launch_rowinfo(structure_of(call.t64), call.n, call.a_nnz, call.lim, call.row_nz,
                                 d_row_ip, call.ctr->sym_counts,
                                 &call.ctr->total_ip, nullptr, call.perm, &call.ctr->long_rows,
                                 call.s);
  if (e != cudaSuccess) return call.cuda_fail(e);
  if ((st = call.fetch_counters())) return st;
  if (total) *total = (int64_t)call.h.total_ip;
  return NSPB_OK;
}

}  // extern "C"
