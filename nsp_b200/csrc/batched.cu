// Batched products C[p] = A[p]·B[p] through one pipeline.
//
// The reference has no batched entry: an AMG setup calls the product once per
// Galerkin step from the host (src/spspmpi.cu:266-313 per call), each call
// creating streams, allocating scratch and synchronising 4-6 times. Here the
// rows of all products form one row space (product p owns the global rows
// [row_off[p], row_off[p+1])), and every phase runs once over it: one launch
// per phase and bin, the bins a single work queue across products, two host
// synchronisations in total. The kernels read each row's operands through a
// device table of per-product descriptors (A's and B's arrays where they lie,
// B's column count) and a row-to-product map, so no operand is copied; C is
// written into one allocation per group, each product's C a view of it, with
// per-product row pointers taken from the group's row pointer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "spgemm_host.h"

namespace nspb {

// The product of every global row: blockIdx.y is the product.
__global__ void k_fill_rows(const int *__restrict__ row_off, int *__restrict__ prod_of_row) {
  const int p = blockIdx.y;
  const int r0 = row_off[p], r1 = row_off[p + 1];
  for (int r = r0 + blockIdx.x * blockDim.x + threadIdx.x; r < r1; r += gridDim.x * blockDim.x)
    prod_of_row[r] = p;
}

// Per-product row pointers (product p's at out_rpt + row_off[p] + p) from the
// group's row pointer.
__global__ void k_split_rows(const int *__restrict__ crpt, const int *__restrict__ row_off,
                             int *__restrict__ out_rpt) {
  const int p = blockIdx.y;
  const int r0 = row_off[p], n = row_off[p + 1] - r0;
  const int c0 = crpt[r0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
    out_rpt[r0 + p + i] = crpt[r0 + i] - c0;
}

// starts[p] = crpt[row_off[p]] for p <= m (row_off[m] = all rows).
__global__ void k_gather_starts(const int *__restrict__ crpt, const int *__restrict__ row_off,
                                int m, int *__restrict__ starts) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= m; p += gridDim.x * blockDim.x)
    starts[p] = crpt[row_off[p]];
}

// Blocks per product on the x axis of the 2-D grids: enough to fill the GPU
// for the largest product of the group.
static dim3 grid2(long long largest, int m) {
  long long g = (largest + 255) / 256;
  const long long cap = std::max<long long>(1, (long long)dev_info().sms * 8);
  return dim3((unsigned)std::max<long long>(1, std::min(g, cap)), (unsigned)m);
}

static int grid_cap(long long n) {
  long long g = (n + 255) / 256;
  const long long cap = (long long)dev_info().sms * 16;
  return (int)std::max<long long>(1, std::min(g, cap));
}

}  // namespace nspb

using namespace nspb;

// Host-side description of one group's product table and the offsets of one
// device block holding it: the per-product operands, each product's first
// global row, the product of every global row, the group's row pointer and
// the per-product starts in C.
struct TableHost {
  int count = 0;
  bool f32 = false;
  long long rows = 0, a_nnz = 0, max_rows = 0;
  int max_ncols = 0, max_brows = 0;
  std::vector<Operands<double>> ops;  // value pointers of fp32 operands stored as-is
  std::vector<int> row_off;
  size_t o_ops = 0, o_roff = 0, o_por = 0, o_crp = 0, o_st = 0, bytes = 0;
};

static int table_layout(int count, const nspb_csr_in *A, const nspb_csr_in *B, bool f32,
                        TableHost &h) {
  h.count = count;
  h.f32 = f32;
  h.ops.resize(count);
  h.row_off.resize(count + 1);
  for (int p = 0; p < count; ++p) {
    const nspb_csr_in &a = A[p], &b = B[p];
    if (a.nrows < 0 || a.ncols != b.nrows || b.ncols < 0 || a.nnz < 0 || b.nnz < 0 ||
        (a.nrows > 0 && !a.rowptr) || (b.nrows > 0 && !b.rowptr) ||
        (a.nnz > 0 && (!a.col || !a.val)) || (b.nnz > 0 && (!b.col || !b.val)))
      return NSPB_ERR_INVALID;
    if (a.nnz > INT32_MAX || b.nnz > INT32_MAX) return NSPB_ERR_INVALID;
    if ((a.nnz > 0 && a.val_type != (f32 ? NSPB_F32 : NSPB_F64)) ||
        (b.nnz > 0 && b.val_type != (f32 ? NSPB_F32 : NSPB_F64)))
      return NSPB_ERR_INVALID;
    Operands<double> o;
    o.arpt = a.rowptr;
    o.acol = a.col;
    o.aval = static_cast<const double *>(a.val);
    o.brpt = b.rowptr;
    o.bcol = b.col;
    o.bval = static_cast<const double *>(b.val);
    o.ncols = b.ncols;
    o.brows = b.nrows;
    h.ops[p] = o;
    h.row_off[p] = (int)h.rows;
    h.rows += a.nrows;
    h.a_nnz += a.nnz;
    h.max_rows = std::max<long long>(h.max_rows, a.nrows);
    h.max_ncols = std::max(h.max_ncols, b.ncols);
    h.max_brows = std::max(h.max_brows, b.nrows);
    if (h.rows >= INT32_MAX) return NSPB_ERR_OVERFLOW;
  }
  h.row_off[count] = (int)h.rows;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  h.o_ops = off; off = al(off + sizeof(Operands<double>) * count);
  h.o_roff = off; off = al(off + 4 * (size_t)(count + 1));
  h.o_por = off; off = al(off + 4 * (size_t)std::max<long long>(h.rows, 1));
  h.o_crp = off; off = al(off + 4 * (size_t)(h.rows + 1));
  h.o_st = off; off = al(off + 4 * (size_t)(count + 1));
  h.bytes = off;
  return NSPB_OK;
}

// Descriptors and row offsets to the device (`host` keeps the staging bytes
// alive until the copy has run), then the row-to-product map.
static cudaError_t table_build(const TableHost &h, char *ws, std::vector<char> &host,
                               cudaStream_t s) {
  host.assign(h.o_por, 0);
  std::memcpy(host.data() + h.o_ops, h.ops.data(), sizeof(Operands<double>) * h.count);
  std::memcpy(host.data() + h.o_roff, h.row_off.data(), 4 * (size_t)(h.count + 1));
  cudaError_t e = cudaMemcpyAsync(ws, host.data(), h.o_por, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  if (h.rows > 0)
    k_fill_rows<<<grid2(h.max_rows, h.count), 256, 0, s>>>(
        reinterpret_cast<const int *>(ws + h.o_roff), reinterpret_cast<int *>(ws + h.o_por));
  return cudaGetLastError();
}

// The group as a call sees it.
static void table_of(const TableHost &h, char *ws, Call &call) {
  ProdTable<double> d;
  d.ops = reinterpret_cast<const Operands<double> *>(ws + h.o_ops);
  d.prod_of_row = reinterpret_cast<const int *>(ws + h.o_por);
  d.row_off = reinterpret_cast<const int *>(ws + h.o_roff);
  ProdTable<float> f;
  f.ops = reinterpret_cast<const Operands<float> *>(ws + h.o_ops);
  f.prod_of_row = d.prod_of_row;
  f.row_off = d.row_off;
  ProdInfo info;
  info.n = (int)h.rows;
  info.max_ncols = h.max_ncols;
  info.nprod = h.count;
  info.max_brows = h.max_brows;
  call.set_table(d, f, info, h.a_nnz);
}

static void table_split(const TableHost &h, char *ws, int *rp_all, cudaStream_t s) {
  k_split_rows<<<grid2(h.max_rows + 1, h.count), 256, 0, s>>>(
      reinterpret_cast<const int *>(ws + h.o_crp), reinterpret_cast<const int *>(ws + h.o_roff),
      rp_all);
}

// First C entry of every product (p <= count), read back to the host.
static cudaError_t table_starts(const TableHost &h, char *ws, std::vector<int> &starts,
                                cudaStream_t s) {
  int *d = reinterpret_cast<int *>(ws + h.o_st);
  k_gather_starts<<<grid_cap(h.count + 1), 256, 0, s>>>(
      reinterpret_cast<const int *>(ws + h.o_crp), reinterpret_cast<const int *>(ws + h.o_roff),
      h.count, d);
  cudaError_t e = cudaGetLastError();
  starts.assign(h.count + 1, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(starts.data(), d, 4 * (size_t)(h.count + 1), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

static void table_views(const TableHost &h, const nspb_csr_in *A, const nspb_csr_in *B,
                        const std::vector<int> &starts, int *rp_all, int *ccol, double *cval,
                        nspb_csr_out *C) {
  for (int p = 0; p < h.count; ++p) {
    C[p].nrows = A[p].nrows;
    C[p].ncols = B[p].ncols;
    C[p].nnz = starts[p + 1] - starts[p];
    C[p].rowptr = rp_all + h.row_off[p] + p;
    C[p].col = ccol + starts[p];
    C[p].val = cval + starts[p];
    C[p].capacity = C[p].nnz;
  }
}

// Statistics of a group of products added into those of the call.
static void add_stats(nspb_stats &t, const nspb_stats &g) {
  t.intprod += g.intprod;
  t.nnz += g.nnz;
  t.launches += g.launches;
  t.rows_redone += g.rows_redone;
  t.max_row_err = std::max(t.max_row_err, g.max_row_err);
  for (int b = 0; b < 16; ++b) {
    t.sym_bins[b] += g.sym_bins[b];
    t.num_bins[b] += g.num_bins[b];
  }
  t.b_sorted = g.b_sorted;
  t.entry_map += g.entry_map;  // groups whose numeric phase ran from entry maps
  t.ms_rowinfo += g.ms_rowinfo;
  t.ms_symbolic += g.ms_symbolic;
  t.ms_scan += g.ms_scan;
  t.ms_numeric += g.ms_numeric;
}

// One group of products through one pipeline. On success C[p] are views into
// one allocation (values, columns, row pointers), whose base pointer is
// appended to owners.
static int batched_group(int count, const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                         const nspb_opts &o, nspb_stats *stats, void **owners, int *n_owners) {
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  TableHost h;
  int st = table_layout(count, A, B, fp32_inputs(o.precision), h);
  if (st) return st;
  Call call;
  if ((st = call.init(&A[0], &B[0], &o))) return st;
  char *ws = nullptr;
  if ((st = scratch_alloc(reinterpret_cast<void **>(&ws), h.bytes, s))) return st;
  std::vector<char> host;
  cudaError_t e = table_build(h, ws, host, s);
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    cudaStreamSynchronize(s);
    scratch_free(ws, s);
    return NSPB_ERR_CUDA;
  }
  table_of(h, ws, call);
  int *crp = reinterpret_cast<int *>(ws + h.o_crp);
  int64_t nnz = 0;
  int *ccol = nullptr, *rp_all = nullptr;
  double *cval = nullptr;
  // C's values, columns and row pointers in one allocation, in that order
  // (each part starts on a 16-byte boundary)
  char *cbase = nullptr;
  st = call.symbolic(crp, &nnz);
  if (!st) {
    const size_t o_col = ((size_t)nnz * 8 + 15) & ~(size_t)15;
    const size_t o_rp = (o_col + (size_t)nnz * 4 + 15) & ~(size_t)15;
    st = alloc_out(reinterpret_cast<void **>(&cbase), o_rp + 4 * (size_t)(h.rows + count));
    if (!st) {
      cval = reinterpret_cast<double *>(cbase);
      ccol = reinterpret_cast<int *>(cbase + o_col);
      rp_all = reinterpret_cast<int *>(cbase + o_rp);
    }
  }
  if (!st) st = call.numeric(crp, ccol, cval);
  if (!st) st = call.finish(stats);
  std::vector<int> starts;
  if (!st) {
    table_split(h, ws, rp_all, s);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = table_starts(h, ws, starts, s);
    if (e != cudaSuccess) {
      g_last_cuda = (int)e;
      cudaGetLastError();
      st = NSPB_ERR_CUDA;
    }
  }
  cudaStreamSynchronize(s);
  scratch_free(ws, s);
  if (st) {
    if (cbase) cudaFree(cbase);
    return st;
  }
  table_views(h, A, B, starts, rp_all, ccol, cval, C);
  owners[(*n_owners)++] = cbase;
  return NSPB_OK;
}

// Products are grouped so that each group's intermediate products (an upper
// bound of its nnz(C)) stay below kGroupIntprod, estimated as
// nnz(A)*nnz(B)/rows(B); a group that still overflows int32 is halved.
constexpr double kGroupIntprod = 1.2e9;

static int batched_range(int first, int count, const nspb_csr_in *A, const nspb_csr_in *B,
                         nspb_csr_out *C, const nspb_opts &o, nspb_stats *stats, void **owners,
                         int *n_owners) {
  nspb_stats gs;
  std::memset(&gs, 0, sizeof(gs));
  int st = batched_group(count, A + first, B + first, C + first, o, &gs, owners, n_owners);
  if (!st) add_stats(*stats, gs);
  if (st == NSPB_ERR_OVERFLOW && count > 1) {
    const int h = count / 2;
    st = batched_range(first, h, A, B, C, o, stats, owners, n_owners);
    if (!st) st = batched_range(first + h, count - h, A, B, C, o, stats, owners, n_owners);
  }
  return st;
}

extern "C" int nspb_spgemm_batched(int count, const nspb_csr_in *A, const nspb_csr_in *B,
                                   nspb_csr_out *C, const nspb_opts *opts, nspb_stats *stats,
                                   void **owners, int32_t *n_owners) {
  if (count < 0 || (count > 0 && (!A || !B || !C || !owners || !n_owners)))
    return NSPB_ERR_INVALID;
  *n_owners = 0;
  if (count == 0) return NSPB_OK;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  int n_own = 0;
  int first = 0;
  nspb_stats total;
  std::memset(&total, 0, sizeof(total));
  while (first < count) {
    double est = 0.0;
    int last = first;
    do {
      const double rb = B[last].nrows > 0 ? (double)B[last].nrows : 1.0;
      est += (double)A[last].nnz * (double)B[last].nnz / rb;
      ++last;
    } while (last < count &&
             (o.batch_max_products <= 0 || last - first < o.batch_max_products) &&
             est + (double)A[last].nnz * (double)B[last].nnz /
                       (B[last].nrows > 0 ? (double)B[last].nrows : 1.0) <=
                 kGroupIntprod);
    nspb_stats gs;
    std::memset(&gs, 0, sizeof(gs));
    const int st = batched_range(first, last - first, A, B, C, o, &gs, owners, &n_own);
    if (st) {
      cudaStreamSynchronize(static_cast<cudaStream_t>(o.stream));
      for (int q = 0; q < n_own; ++q) cudaFree(owners[q]);
      *n_owners = 0;
      return st;
    }
    add_stats(total, gs);
    first = last;
  }
  *n_owners = n_own;
  if (stats) *stats = total;
  return NSPB_OK;
}

// ---- plans: the numeric phase of a fixed structure replayed from a CUDA graph --
namespace nspb {

// One group of a plan: one product, or several through a product table.
struct PlanGroup {
  bool multi = false;          // several products (a table)
  TableHost h;                 // the table's layout (multi)
  Call call;                   // the products whose numeric phase is captured
  char *ws_tab = nullptr;      // the table and the group's row pointer (multi)
  char *ws_call = nullptr;     // the call's scratch (bins, permutation, counters)
  int *crp = nullptr;          // C's row pointer of a single product
  int *rp_all = nullptr;       // per-product row pointers (multi)
  int *ccol = nullptr;
  double *cval = nullptr;
  long long nnz = 0;
  ~PlanGroup() {
    call.s = nullptr;  // the capture stream is gone: the call's pool blocks go back on the legacy stream
    for (void *p : {(void *)ws_tab, (void *)ws_call, (void *)crp, (void *)rp_all, (void *)ccol,
                    (void *)cval})
      if (p) cudaFree(p);
  }
};

}  // namespace nspb

struct nspb_plan_s {
  bool check = false;          // execute reports the device error words
  std::vector<std::unique_ptr<nspb::PlanGroup>> groups;
  int *h_err = nullptr;        // pinned: one error word per group
  cudaStream_t cs = nullptr;   // capture stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~nspb_plan_s() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cs) cudaStreamDestroy(cs);
    if (h_err) cudaFreeHost(h_err);
    groups.clear();  // cudaFree waits for an execution still in flight
  }
};

namespace {

int plan_fail(cudaError_t e) {
  g_last_cuda = (int)e;
  cudaGetLastError();
  return NSPB_ERR_CUDA;
}

template <typename T>
int dev_alloc(T **p, size_t count) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    return NSPB_ERR_ALLOC;
  }
  return NSPB_OK;
}

// The numeric phase of a group as launched on every execution: counters
// zeroed, then the bin kernels, which read the operands' current values
// where they lie (structure and C's row pointers do not change).
int group_numeric(PlanGroup &G, cudaStream_t s) {
  G.call.s = s;
  if (G.call.n == 0) return NSPB_OK;  // no rows: no scratch, nothing to compute
  cudaError_t e = cudaMemsetAsync(G.call.ctr, 0, sizeof(DevCounters), s);
  if (e != cudaSuccess) return plan_fail(e);
  const int *crp = G.multi ? reinterpret_cast<int *>(G.ws_tab + G.h.o_crp) : G.crp;
  return G.call.numeric(crp, G.ccol, G.cval);
}


// Symbolic phase, C's arrays and one checked numeric pass of the products
// [0, count); the C views are filled.
int group_create(int count, const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                 const nspb_opts &o, nspb_stats *stats, std::unique_ptr<PlanGroup> &out) {
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  std::unique_ptr<PlanGroup> G(new PlanGroup);
  G->multi = count > 1;
  int st;
  if ((st = G->call.init(&A[0], &B[0], &o))) return st;
  if (G->multi) {
    if ((st = table_layout(count, A, B, fp32_inputs(o.precision), G->h))) return st;
    if ((st = dev_alloc(&G->ws_tab, G->h.bytes))) return st;
    std::vector<char> host;
    cudaError_t e = table_build(G->h, G->ws_tab, host, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // `host` is released below
    if (e != cudaSuccess) return plan_fail(e);
    table_of(G->h, G->ws_tab, G->call);
  }
  const size_t wb = G->call.scratch_bytes();
  if ((st = dev_alloc(&G->ws_call, wb))) return st;
  G->call.ext_ws = G->ws_call;
  G->call.ext_bytes = wb;
  int *crp = nullptr;
  if (G->multi) {
    crp = reinterpret_cast<int *>(G->ws_tab + G->h.o_crp);
  } else {
    if ((st = dev_alloc(&G->crp, (size_t)A[0].nrows + 1))) return st;
    crp = G->crp;
  }
  int64_t nnz = 0;
  if ((st = G->call.symbolic(crp, &nnz))) return st;
  G->nnz = nnz;
  if ((st = dev_alloc(&G->ccol, (size_t)nnz)) || (st = dev_alloc(&G->cval, (size_t)nnz))) return st;
  if (G->multi) {
    if ((st = dev_alloc(&G->rp_all, (size_t)(G->h.rows + count)))) return st;
    table_split(G->h, G->ws_tab, G->rp_all, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return plan_fail(e);
  }
  // one pass on the caller's stream (fills C and the launch caches), checked;
  // the pass zeroes the device counters, so the symbolic counts are kept
  const DevCounters sym = G->call.h;
  if ((st = group_numeric(*G, s))) return st;
  if (G->call.n > 0 && (st = G->call.fetch_counters())) return st;  // error word, redo counts
  DevCounters &hc = G->call.h;
  hc.total_nnz = sym.total_nnz;
  std::memcpy(hc.sym_counts, sym.sym_counts, sizeof(hc.sym_counts));
  std::memcpy(hc.num_counts, sym.num_counts, sizeof(hc.num_counts));
  nspb_stats gs;
  std::memset(&gs, 0, sizeof(gs));
  const nspb_opts keep = G->call.opts;
  G->call.opts.check_errors = 0;  // finish: no second read of the counters
  G->call.opts.precision = NSPB_PREC_FP64;
  st = G->call.finish(&gs);
  G->call.opts = keep;
  if (st) return st;
  if (keep.precision == NSPB_PREC_FP32_COMP) {
    gs.rows_redone = hc.redo_count;
    gs.max_row_err = comp_bound(hc.max_comp_deg);
  }
  if (stats) add_stats(*stats, gs);
  if (G->multi) {
    std::vector<int> starts;
    cudaError_t e = table_starts(G->h, G->ws_tab, starts, s);
    if (e != cudaSuccess) return plan_fail(e);
    table_views(G->h, A, B, starts, G->rp_all, G->ccol, G->cval, C);
  } else {
    C[0].nrows = A[0].nrows;
    C[0].ncols = B[0].ncols;
    C[0].nnz = nnz;
    C[0].rowptr = G->crp;
    C[0].col = G->ccol;
    C[0].val = G->cval;
    C[0].capacity = nnz;
  }
  out = std::move(G);
  return NSPB_OK;
}

// Groups of [first, first+count): halved while the block-diagonal product
// does not fit int32.
int plan_range(nspb_plan_s &P, int first, int count, const nspb_csr_in *A,
               const nspb_csr_in *B, nspb_csr_out *C, const nspb_opts &o, nspb_stats *stats) {
  std::unique_ptr<PlanGroup> G;
  nspb_stats gs;
  std::memset(&gs, 0, sizeof(gs));
  int st = group_create(count, A + first, B + first, C + first, o, &gs, G);
  if (st == NSPB_ERR_OVERFLOW && count > 1) {
    const int h = count / 2;
    st = plan_range(P, first, h, A, B, C, o, stats);
    if (!st) st = plan_range(P, first + h, count - h, A, B, C, o, stats);
    return st;
  }
  if (st) return st;
  if (stats) add_stats(*stats, gs);
  P.groups.push_back(std::move(G));
  return NSPB_OK;
}

}  // namespace

extern "C" int nspb_plan_create(int count, const nspb_csr_in *A, const nspb_csr_in *B,
                                nspb_csr_out *C, const nspb_opts *opts, nspb_stats *stats,
                                nspb_plan *plan) {
  if (!plan || count <= 0 || !A || !B || !C) return NSPB_ERR_INVALID;
  *plan = nullptr;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  o.timing = 0;
  std::unique_ptr<nspb_plan_s> P(new nspb_plan_s);
  P->check = o.check_errors != 0;
  nspb_stats total;
  std::memset(&total, 0, sizeof(total));
  // the grouping of nspb_spgemm_batched
  int st = NSPB_OK;
  for (int first = 0; first < count && !st;) {
    double est = 0.0;
    int last = first;
    do {
      const double rb = B[last].nrows > 0 ? (double)B[last].nrows : 1.0;
      est += (double)A[last].nnz * (double)B[last].nnz / rb;
      ++last;
    } while (last < count &&
             (o.batch_max_products <= 0 || last - first < o.batch_max_products) &&
             est + (double)A[last].nnz * (double)B[last].nnz /
                       (B[last].nrows > 0 ? (double)B[last].nrows : 1.0) <=
                 kGroupIntprod);
    st = plan_range(*P, first, last - first, A, B, C, o, &total);
    first = last;
  }
  if (st) {
    cudaStreamSynchronize(static_cast<cudaStream_t>(o.stream));
    return st;
  }
  cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(&P->h_err),
                                 sizeof(int) * P->groups.size());
  if (e != cudaSuccess) return plan_fail(e);
  // every group's numeric phase captured once, in order, into one graph
  if ((e = cudaStreamCreateWithFlags(&P->cs, cudaStreamNonBlocking)) != cudaSuccess)
    return plan_fail(e);
  if ((e = cudaStreamBeginCapture(P->cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return plan_fail(e);
  for (auto &G : P->groups)
    if (!st) st = group_numeric(*G, P->cs);
  e = cudaStreamEndCapture(P->cs, &P->graph);  // always leave capture mode
  if (st) return st;
  if (e != cudaSuccess) return plan_fail(e);
  if ((e = cudaGraphInstantiate(&P->exec, P->graph, 0)) != cudaSuccess) return plan_fail(e);
  if (stats) *stats = total;
  *plan = P.release();
  return NSPB_OK;
}

extern "C" int nspb_plan_execute(nspb_plan P, void *stream) {
  if (!P || !P->exec) return NSPB_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaGraphLaunch(P->exec, s);
  if (e != cudaSuccess) return plan_fail(e);
  if (!P->check) return NSPB_OK;
  for (size_t g = 0; g < P->groups.size() && e == cudaSuccess; ++g) {
    P->h_err[g] = 0;
    if (P->groups[g]->call.ctr)  // groups without rows have no counters
      e = cudaMemcpyAsync(P->h_err + g, &P->groups[g]->call.ctr->err, sizeof(int),
                          cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return plan_fail(e);
  for (size_t g = 0; g < P->groups.size(); ++g)
    if (P->h_err[g]) return NSPB_ERR_DEVICE;
  return NSPB_OK;
}

extern "C" int nspb_plan_destroy(nspb_plan P) {
  delete P;
  return NSPB_OK;
}
