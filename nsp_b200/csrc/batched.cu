// Batched products C[p] = A[p]·B[p] through one pipeline.
//
// The reference has no batched entry: an AMG setup calls the product once per
// Galerkin step from the host (src/spspmpi.cu:266-313 per call), each call
// creating streams, allocating scratch and synchronising 4-6 times. Here the
// batch is one block-diagonal product:
//   A_cat = diag(A[0], ..., A[m-1]),  B_cat = diag(B[0], ..., B[m-1])
//   C_cat = A_cat·B_cat = diag(A[0]B[0], ..., A[m-1]B[m-1])
// One kernel copies the operands into the block-diagonal layout (columns of
// A[p] shifted by the first row of B[p] in B_cat, columns of B[p] by its first
// column), the standard pipeline then runs once over all rows of all
// products (one launch per phase and bin; the bins form a single work queue
// across products; two host synchronisations in total), and one kernel
// splits C_cat back into per-product row pointers and columns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "spgemm_host.h"

namespace nspb {

struct CatDesc {
  const int *rpt;
  const int *col;
  const void *val;
  long long row_off;  // first row of this block in the concatenation
  long long nnz_off;  // first entry of this block
  int nrows;
  int col_shift;      // added to every column of this block
};

// The concatenation and split kernels run on a 2-D grid: blockIdx.y is the
// product, blockIdx.x strides over that product's rows or entries, so no item
// has to search for its product.
template <typename VT>
__global__ void k_cat_entries(const CatDesc *__restrict__ d, int *__restrict__ col,
                              VT *__restrict__ val) {
  const CatDesc q = d[blockIdx.y];
  const long long n = (long long)(q.nrows > 0 ? q.rpt[q.nrows] - q.rpt[0] : 0);
  const long long e0 = q.nrows > 0 ? q.rpt[0] : 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    col[q.nnz_off + e] = q.col[e0 + e] + q.col_shift;
    val[q.nnz_off + e] = static_cast<const VT *>(q.val)[e0 + e];
  }
}

__global__ void k_cat_rows(const CatDesc *__restrict__ d, long long total, long long nnz_total,
                           int *__restrict__ rpt) {
  const CatDesc q = d[blockIdx.y];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < q.nrows;
       i += (long long)gridDim.x * blockDim.x)
    rpt[q.row_off + i] = (int)(q.nnz_off + (q.rpt[i] - q.rpt[0]));
  if (blockIdx.y == 0 && blockIdx.x == 0 && threadIdx.x == 0) rpt[total] = (int)nnz_total;
}

// Per-product row pointers (product p's at out_rpt + row_off[p] + p) and the
// column shift undone in place.
__global__ void k_split(const int *__restrict__ crpt, const long long *__restrict__ row_off,
                        const int *__restrict__ shift, int *__restrict__ out_rpt,
                        int *__restrict__ ccol) {
  const int p = blockIdx.y;
  const long long r0 = row_off[p], n = row_off[p + 1] - r0;
  const int c0 = crpt[r0], c1 = crpt[r0 + n], sh = shift[p];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (long long)gridDim.x * blockDim.x)
    out_rpt[r0 + p + i] = crpt[r0 + i] - c0;
  for (long long t = c0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; t < c1;
       t += (long long)gridDim.x * blockDim.x)
    ccol[t] -= sh;
}

// starts[p] = crpt[row_off[p]] for p <= m (row_off[m] = all rows).
__global__ void k_gather_starts(const int *__restrict__ crpt, const long long *__restrict__ row_off,
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

// Host-side layout of the block-diagonal operands of `count` products and the
// offsets of one device block holding descriptors, offsets, the concatenated
// A and B and C_cat's row pointer.
struct CatHost {
  int count = 0;
  bool f32 = false;
  long long rows_a = 0, rows_b = 0, cols_b = 0, nnz_a = 0, nnz_b = 0;
  long long max_ra = 0, max_rb = 0, max_na = 0, max_nb = 0;
  std::vector<CatDesc> da, db;
  std::vector<long long> a_rows, a_nnz, b_rows, b_nnz;
  std::vector<int> cshift;
  size_t o_da, o_db, o_ar, o_an, o_br, o_bn, o_sh, o_arp, o_acl, o_avl, o_brp, o_bcl, o_bvl,
      o_crp, o_st, bytes;
};

static int cat_layout(int count, const nspb_csr_in *A, const nspb_csr_in *B, bool f32,
                      CatHost &h) {
  h.count = count;
  h.f32 = f32;
  h.da.resize(count);
  h.db.resize(count);
  h.a_rows.resize(count + 1);
  h.a_nnz.resize(count + 1);
  h.b_rows.resize(count + 1);
  h.b_nnz.resize(count + 1);
  h.cshift.resize(count);
  for (int p = 0; p < count; ++p) {
    const nspb_csr_in &a = A[p], &b = B[p];
    if (a.nrows < 0 || a.ncols != b.nrows || b.ncols < 0 || a.nnz < 0 || b.nnz < 0 ||
        (a.nrows > 0 && !a.rowptr) || (b.nrows > 0 && !b.rowptr) ||
        (a.nnz > 0 && (!a.col || !a.val)) || (b.nnz > 0 && (!b.col || !b.val)))
      return NSPB_ERR_INVALID;
    if ((a.nnz > 0 && a.val_type != (f32 ? NSPB_F32 : NSPB_F64)) ||
        (b.nnz > 0 && b.val_type != (f32 ? NSPB_F32 : NSPB_F64)))
      return NSPB_ERR_INVALID;
    h.da[p] = CatDesc{a.rowptr, a.col, a.val, h.rows_a, h.nnz_a, a.nrows, (int)h.rows_b};
    h.db[p] = CatDesc{b.rowptr, b.col, b.val, h.rows_b, h.nnz_b, b.nrows, (int)h.cols_b};
    h.cshift[p] = (int)h.cols_b;
    h.a_rows[p] = h.rows_a;
    h.a_nnz[p] = h.nnz_a;
    h.b_rows[p] = h.rows_b;
    h.b_nnz[p] = h.nnz_b;
    h.rows_a += a.nrows;
    h.nnz_a += a.nnz;
    h.rows_b += b.nrows;
    h.nnz_b += b.nnz;
    h.cols_b += b.ncols;
    h.max_ra = std::max<long long>(h.max_ra, a.nrows);
    h.max_rb = std::max<long long>(h.max_rb, b.nrows);
    h.max_na = std::max<long long>(h.max_na, a.nnz);
    h.max_nb = std::max<long long>(h.max_nb, b.nnz);
  }
  h.a_rows[count] = h.rows_a;
  h.a_nnz[count] = h.nnz_a;
  h.b_rows[count] = h.rows_b;
  h.b_nnz[count] = h.nnz_b;
  if (h.rows_a >= INT32_MAX || h.rows_b >= INT32_MAX || h.cols_b >= INT32_MAX ||
      h.nnz_a > INT32_MAX || h.nnz_b > INT32_MAX)
    return NSPB_ERR_OVERFLOW;
  const size_t vsz = f32 ? 4 : 8;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  h.o_da = off; off = al(off + sizeof(CatDesc) * count);
  h.o_db = off; off = al(off + sizeof(CatDesc) * count);
  h.o_ar = off; off = al(off + 8 * (count + 1));
  h.o_an = off; off = al(off + 8 * (count + 1));
  h.o_br = off; off = al(off + 8 * (count + 1));
  h.o_bn = off; off = al(off + 8 * (count + 1));
  h.o_sh = off; off = al(off + 4 * count);
  h.o_arp = off; off = al(off + 4 * (h.rows_a + 1));
  h.o_acl = off; off = al(off + 4 * h.nnz_a);
  h.o_avl = off; off = al(off + vsz * h.nnz_a);
  h.o_brp = off; off = al(off + 4 * (h.rows_b + 1));
  h.o_bcl = off; off = al(off + 4 * h.nnz_b);
  h.o_bvl = off; off = al(off + vsz * h.nnz_b);
  h.o_crp = off; off = al(off + 4 * (h.rows_a + 1));
  h.o_st = off; off = al(off + 4 * (count + 1));
  h.bytes = off;
  return NSPB_OK;
}

// Columns and values of every product into the block-diagonal arrays.
static void cat_entries(const CatHost &h, char *ws, cudaStream_t s) {
  const CatDesc *dda = reinterpret_cast<const CatDesc *>(ws + h.o_da);
  const CatDesc *ddb = reinterpret_cast<const CatDesc *>(ws + h.o_db);
  int *acl = reinterpret_cast<int *>(ws + h.o_acl), *bcl = reinterpret_cast<int *>(ws + h.o_bcl);
  if (h.f32) {
    k_cat_entries<float><<<grid2(h.max_na, h.count), 256, 0, s>>>(
        dda, acl, reinterpret_cast<float *>(ws + h.o_avl));
    k_cat_entries<float><<<grid2(h.max_nb, h.count), 256, 0, s>>>(
        ddb, bcl, reinterpret_cast<float *>(ws + h.o_bvl));
  } else {
    k_cat_entries<double><<<grid2(h.max_na, h.count), 256, 0, s>>>(
        dda, acl, reinterpret_cast<double *>(ws + h.o_avl));
    k_cat_entries<double><<<grid2(h.max_nb, h.count), 256, 0, s>>>(
        ddb, bcl, reinterpret_cast<double *>(ws + h.o_bvl));
  }
}

// Descriptors to the device (`host` keeps the staging bytes alive until the
// copy has run), then the row pointers and entries of the concatenation.
static cudaError_t cat_build(const CatHost &h, char *ws, std::vector<char> &host,
                             cudaStream_t s) {
  host.assign(h.o_arp, 0);
  std::memcpy(host.data() + h.o_da, h.da.data(), sizeof(CatDesc) * h.count);
  std::memcpy(host.data() + h.o_db, h.db.data(), sizeof(CatDesc) * h.count);
  std::memcpy(host.data() + h.o_ar, h.a_rows.data(), 8 * (h.count + 1));
  std::memcpy(host.data() + h.o_an, h.a_nnz.data(), 8 * (h.count + 1));
  std::memcpy(host.data() + h.o_br, h.b_rows.data(), 8 * (h.count + 1));
  std::memcpy(host.data() + h.o_bn, h.b_nnz.data(), 8 * (h.count + 1));
  std::memcpy(host.data() + h.o_sh, h.cshift.data(), 4 * h.count);
  cudaError_t e = cudaMemcpyAsync(ws, host.data(), h.o_arp, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  const CatDesc *dda = reinterpret_cast<const CatDesc *>(ws + h.o_da);
  const CatDesc *ddb = reinterpret_cast<const CatDesc *>(ws + h.o_db);
  k_cat_rows<<<grid2(h.max_ra, h.count), 256, 0, s>>>(dda, h.rows_a, h.nnz_a,
                                                       reinterpret_cast<int *>(ws + h.o_arp));
  k_cat_rows<<<grid2(h.max_rb, h.count), 256, 0, s>>>(ddb, h.rows_b, h.nnz_b,
                                                       reinterpret_cast<int *>(ws + h.o_brp));
  cat_entries(h, ws, s);
  return cudaGetLastError();
}

static nspb_csr_in cat_in(const CatHost &h, char *ws, bool is_a) {
  const int32_t vt = h.f32 ? NSPB_F32 : NSPB_F64;
  if (is_a)
    return nspb_csr_in{(int32_t)h.rows_a, (int32_t)h.rows_b, h.nnz_a,
                       reinterpret_cast<int *>(ws + h.o_arp), reinterpret_cast<int *>(ws + h.o_acl),
                       ws + h.o_avl, vt, 0};
  return nspb_csr_in{(int32_t)h.rows_b, (int32_t)h.cols_b, h.nnz_b,
                     reinterpret_cast<int *>(ws + h.o_brp), reinterpret_cast<int *>(ws + h.o_bcl),
                     ws + h.o_bvl, vt, 0};
}

// Per-product row pointers into rp_all and C_cat's columns shifted back.
static void cat_split(const CatHost &h, char *ws, long long nnz_c, int *rp_all, int *ccol,
                      cudaStream_t s) {
  const long long per = std::max<long long>(nnz_c / std::max(h.count, 1) * 4, 1 << 16);
  k_split<<<grid2(per, h.count), 256, 0, s>>>(
      reinterpret_cast<const int *>(ws + h.o_crp), reinterpret_cast<const long long *>(ws + h.o_ar),
      reinterpret_cast<const int *>(ws + h.o_sh), rp_all, ccol);
}

// First C_cat entry of every product (p <= count), read back to the host.
static cudaError_t cat_starts(const CatHost &h, char *ws, std::vector<int> &starts,
                              cudaStream_t s) {
  int *d = reinterpret_cast<int *>(ws + h.o_st);
  k_gather_starts<<<grid_cap(h.count + 1), 256, 0, s>>>(
      reinterpret_cast<const int *>(ws + h.o_crp), reinterpret_cast<const long long *>(ws + h.o_ar),
      h.count, d);
  cudaError_t e = cudaGetLastError();
  starts.assign(h.count + 1, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(starts.data(), d, 4 * (h.count + 1), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

static void cat_views(const CatHost &h, const nspb_csr_in *A, const nspb_csr_in *B,
                      const std::vector<int> &starts, int *rp_all, int *ccol, double *cval,
                      nspb_csr_out *C) {
  for (int p = 0; p < h.count; ++p) {
    C[p].nrows = A[p].nrows;
    C[p].ncols = B[p].ncols;
    C[p].nnz = starts[p + 1] - starts[p];
    C[p].rowptr = rp_all + h.a_rows[p] + p;
    C[p].col = ccol + starts[p];
    C[p].val = cval + starts[p];
    C[p].capacity = C[p].nnz;
  }
}

// One group of products as one block-diagonal product. On success C[p] are
// views into two allocations (C_cat col/val) plus the row-pointer block; the
// three base pointers are appended to owners.
static int batched_group(int count, const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                         const nspb_opts &o, nspb_stats *stats, void **owners, int *n_owners) {
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  CatHost h;
  int st = cat_layout(count, A, B, fp32_inputs(o.precision), h);
  if (st) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NSPB_ERR_NO_DEVICE;
  }
  char *ws = nullptr;
  if ((st = scratch_alloc(reinterpret_cast<void **>(&ws), h.bytes, s))) return st;
  std::vector<char> host;
  cudaError_t e = cat_build(h, ws, host, s);
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    cudaStreamSynchronize(s);
    scratch_free(ws, s);
    return NSPB_ERR_CUDA;
  }
  // the product of the block-diagonal operands, C_cat arrays allocated here
  const nspb_csr_in Acat = cat_in(h, ws, true), Bcat = cat_in(h, ws, false);
  nspb_csr_out Ccat;
  std::memset(&Ccat, 0, sizeof(Ccat));
  Ccat.rowptr = reinterpret_cast<int *>(ws + h.o_crp);
  st = nspb_spgemm(&Acat, &Bcat, &Ccat, &o, stats);
  if (st) {
    cudaStreamSynchronize(s);
    scratch_free(ws, s);
    return st;
  }
  int *rp_all = nullptr;
  st = alloc_out(reinterpret_cast<void **>(&rp_all), 4 * (size_t)(h.rows_a + count));
  std::vector<int> starts;
  if (!st) {
    cat_split(h, ws, Ccat.nnz, rp_all, Ccat.col, s);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cat_starts(h, ws, starts, s);
    if (e != cudaSuccess) {
      g_last_cuda = (int)e;
      st = NSPB_ERR_CUDA;
    }
  }
  scratch_free(ws, s);
  if (st) {
    cudaStreamSynchronize(s);
    if (rp_all) cudaFree(rp_all);
    cudaFree(Ccat.col);
    cudaFree(Ccat.val);
    return st;
  }
  cat_views(h, A, B, starts, rp_all, Ccat.col, Ccat.val, C);
  owners[(*n_owners)++] = rp_all;
  owners[(*n_owners)++] = Ccat.col;
  owners[(*n_owners)++] = Ccat.val;
  return NSPB_OK;
}

// Products are grouped so that each group's intermediate products (an upper
// bound of its nnz(C)) stay below kGroupIntprod, estimated as
// nnz(A)*nnz(B)/rows(B); a group that still overflows int32 is halved.
constexpr double kGroupIntprod = 1.2e9;

static int batched_range(int first, int count, const nspb_csr_in *A, const nspb_csr_in *B,
                         nspb_csr_out *C, const nspb_opts &o, nspb_stats *stats, void **owners,
                         int *n_owners) {
  int st = batched_group(count, A + first, B + first, C + first, o, stats, owners, n_owners);
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
    total.intprod += gs.intprod;
    total.nnz += gs.nnz;
    total.launches += gs.launches;
    total.rows_redone += gs.rows_redone;
    total.max_row_err = std::max(total.max_row_err, gs.max_row_err);
    for (int b = 0; b < 16; ++b) {
      total.sym_bins[b] += gs.sym_bins[b];
      total.num_bins[b] += gs.num_bins[b];
    }
    total.b_sorted = gs.b_sorted;
    first = last;
  }
  *n_owners = n_own;
  if (stats) *stats = total;
  return NSPB_OK;
}

// ---- plans: the numeric phase of a fixed structure replayed from a CUDA graph --
namespace nspb {

// One group of a plan: one product, or several as one block-diagonal product.
struct PlanGroup {
  bool cat = false;            // block-diagonal operands
  CatHost h;                   // their layout (cat)
  Call call;                   // the product whose numeric phase is captured
  char *ws_cat = nullptr;      // concatenated operands and C_cat's row pointer
  char *ws_call = nullptr;     // the call's scratch (bins, permutation, counters)
  int *crp = nullptr;          // C's row pointer of a single product
  int *rp_all = nullptr;       // per-product row pointers (cat)
  int *ccol = nullptr;
  double *cval = nullptr;
  long long nnz = 0;
  ~PlanGroup() {
    for (void *p : {(void *)ws_cat, (void *)ws_call, (void *)crp, (void *)rp_all, (void *)ccol,
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
// zeroed, operand entries concatenated, bin kernels, split.
int group_numeric(PlanGroup &G, cudaStream_t s) {
  G.call.s = s;
  if (G.call.n == 0) return NSPB_OK;  // no rows: no scratch, nothing to compute
  cudaError_t e = cudaMemsetAsync(G.call.ctr, 0, sizeof(DevCounters), s);
  if (e != cudaSuccess) return plan_fail(e);
  if (G.cat) {
    cat_entries(G.h, G.ws_cat, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return plan_fail(e);
  }
  const int *crp = G.cat ? reinterpret_cast<int *>(G.ws_cat + G.h.o_crp) : G.crp;
  int st = G.call.numeric(crp, G.ccol, G.cval);
  if (st) return st;
  if (G.cat) {
    cat_split(G.h, G.ws_cat, G.nnz, G.rp_all, G.ccol, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return plan_fail(e);
  }
  return NSPB_OK;
}

void add_stats(nspb_stats &t, const nspb_stats &g) {
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
}

// Symbolic phase, C's arrays and one checked numeric pass of the products
// [0, count); the C views are filled.
int group_create(int count, const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                 const nspb_opts &o, nspb_stats *stats, std::unique_ptr<PlanGroup> &out) {
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  std::unique_ptr<PlanGroup> G(new PlanGroup);
  G->cat = count > 1;
  int st;
  nspb_csr_in a = A[0], b = B[0];
  if (G->cat) {
    if ((st = cat_layout(count, A, B, fp32_inputs(o.precision), G->h))) return st;
    if ((st = dev_alloc(&G->ws_cat, G->h.bytes))) return st;
    std::vector<char> host;
    cudaError_t e = cat_build(G->h, G->ws_cat, host, s);
    if (e != cudaSuccess) return plan_fail(e);
    a = cat_in(G->h, G->ws_cat, true);
    b = cat_in(G->h, G->ws_cat, false);
  }
  if ((st = G->call.init(&a, &b, &o))) return st;
  const size_t wb = G->call.scratch_bytes();
  if ((st = dev_alloc(&G->ws_call, wb))) return st;
  G->call.ext_ws = G->ws_call;
  G->call.ext_bytes = wb;
  int *crp = nullptr;
  if (G->cat) {
    crp = reinterpret_cast<int *>(G->ws_cat + G->h.o_crp);
  } else {
    if ((st = dev_alloc(&G->crp, (size_t)a.nrows + 1))) return st;
    crp = G->crp;
  }
  int64_t nnz = 0;
  if ((st = G->call.symbolic(crp, &nnz))) return st;
  G->nnz = nnz;
  if ((st = dev_alloc(&G->ccol, (size_t)nnz)) || (st = dev_alloc(&G->cval, (size_t)nnz))) return st;
  if (G->cat && (st = dev_alloc(&G->rp_all, (size_t)(G->h.rows_a + count)))) return st;
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
  if (G->cat) {
    std::vector<int> starts;
    cudaError_t e = cat_starts(G->h, G->ws_cat, starts, s);
    if (e != cudaSuccess) return plan_fail(e);
    cat_views(G->h, A, B, starts, G->rp_all, G->ccol, G->cval, C);
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
