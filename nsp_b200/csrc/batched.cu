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

// One group of products as one block-diagonal product. On success C[p] are
// views into two allocations (C_cat col/val) plus the row-pointer block; the
// three base pointers are appended to owners.
static int batched_group(int count, const nspb_csr_in *A, const nspb_csr_in *B, nspb_csr_out *C,
                         const nspb_opts &o, nspb_stats *stats, void **owners, int *n_owners) {
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  const bool f32 = o.precision == NSPB_PREC_FP32_COMP;
  const size_t vsz = f32 ? 4 : 8;
  // host-side layout of the block-diagonal operands
  long long rows_a = 0, rows_b = 0, cols_b = 0, nnz_a = 0, nnz_b = 0;
  std::vector<CatDesc> da(count), db(count);
  std::vector<long long> a_rows(count + 1), a_nnz(count + 1), b_rows(count + 1), b_nnz(count + 1);
  std::vector<int> cshift(count);
  for (int p = 0; p < count; ++p) {
    const nspb_csr_in &a = A[p], &b = B[p];
    if (a.nrows < 0 || a.ncols != b.nrows || b.ncols < 0 || a.nnz < 0 || b.nnz < 0 ||
        (a.nrows > 0 && !a.rowptr) || (b.nrows > 0 && !b.rowptr) ||
        (a.nnz > 0 && (!a.col || !a.val)) || (b.nnz > 0 && (!b.col || !b.val)))
      return NSPB_ERR_INVALID;
    if ((a.nnz > 0 && a.val_type != (f32 ? NSPB_F32 : NSPB_F64)) ||
        (b.nnz > 0 && b.val_type != (f32 ? NSPB_F32 : NSPB_F64)))
      return NSPB_ERR_INVALID;
    da[p] = CatDesc{a.rowptr, a.col, a.val, rows_a, nnz_a, a.nrows, (int)rows_b};
    db[p] = CatDesc{b.rowptr, b.col, b.val, rows_b, nnz_b, b.nrows, (int)cols_b};
    cshift[p] = (int)cols_b;
    a_rows[p] = rows_a; a_nnz[p] = nnz_a; b_rows[p] = rows_b; b_nnz[p] = nnz_b;
    rows_a += a.nrows; nnz_a += a.nnz; rows_b += b.nrows; nnz_b += b.nnz; cols_b += b.ncols;
  }
  a_rows[count] = rows_a; a_nnz[count] = nnz_a; b_rows[count] = rows_b; b_nnz[count] = nnz_b;
  if (rows_a >= INT32_MAX || rows_b >= INT32_MAX || cols_b >= INT32_MAX ||
      nnz_a > INT32_MAX || nnz_b > INT32_MAX)
    return NSPB_ERR_OVERFLOW;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NSPB_ERR_NO_DEVICE;
  }
  // one scratch block: descriptors, offsets, concatenated A and B
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  const size_t o_da = off; off = al(off + sizeof(CatDesc) * count);
  const size_t o_db = off; off = al(off + sizeof(CatDesc) * count);
  const size_t o_ar = off; off = al(off + 8 * (count + 1));
  const size_t o_an = off; off = al(off + 8 * (count + 1));
  const size_t o_br = off; off = al(off + 8 * (count + 1));
  const size_t o_bn = off; off = al(off + 8 * (count + 1));
  const size_t o_sh = off; off = al(off + 4 * count);
  const size_t o_arp = off; off = al(off + 4 * (rows_a + 1));
  const size_t o_acl = off; off = al(off + 4 * nnz_a);
  const size_t o_avl = off; off = al(off + vsz * nnz_a);
  const size_t o_brp = off; off = al(off + 4 * (rows_b + 1));
  const size_t o_bcl = off; off = al(off + 4 * nnz_b);
  const size_t o_bvl = off; off = al(off + vsz * nnz_b);
  const size_t o_crp = off; off = al(off + 4 * (rows_a + 1));
  const size_t o_st = off; off = al(off + 4 * (count + 1));
  char *ws = nullptr;
  int st = scratch_alloc(reinterpret_cast<void **>(&ws), off, s);
  if (st) return st;
  std::vector<char> host(o_arp);
  std::memcpy(host.data() + o_da, da.data(), sizeof(CatDesc) * count);
  std::memcpy(host.data() + o_db, db.data(), sizeof(CatDesc) * count);
  std::memcpy(host.data() + o_ar, a_rows.data(), 8 * (count + 1));
  std::memcpy(host.data() + o_an, a_nnz.data(), 8 * (count + 1));
  std::memcpy(host.data() + o_br, b_rows.data(), 8 * (count + 1));
  std::memcpy(host.data() + o_bn, b_nnz.data(), 8 * (count + 1));
  std::memcpy(host.data() + o_sh, cshift.data(), 4 * count);
  cudaError_t e = cudaMemcpyAsync(ws, host.data(), o_arp, cudaMemcpyHostToDevice, s);
  auto D = [&](size_t o_) { return ws + o_; };
  const CatDesc *dda = reinterpret_cast<const CatDesc *>(D(o_da));
  const CatDesc *ddb = reinterpret_cast<const CatDesc *>(D(o_db));
  int *arp = reinterpret_cast<int *>(D(o_arp)), *acl = reinterpret_cast<int *>(D(o_acl));
  int *brp = reinterpret_cast<int *>(D(o_brp)), *bcl = reinterpret_cast<int *>(D(o_bcl));
  int *crp = reinterpret_cast<int *>(D(o_crp));
  const long long *d_ar = reinterpret_cast<const long long *>(D(o_ar));
  if (e == cudaSuccess) {
    long long max_ra = 0, max_rb = 0, max_na = 0, max_nb = 0;
    for (int p = 0; p < count; ++p) {
      max_ra = std::max<long long>(max_ra, A[p].nrows);
      max_rb = std::max<long long>(max_rb, B[p].nrows);
      max_na = std::max<long long>(max_na, A[p].nnz);
      max_nb = std::max<long long>(max_nb, B[p].nnz);
    }
    k_cat_rows<<<grid2(max_ra, count), 256, 0, s>>>(dda, rows_a, nnz_a, arp);
    k_cat_rows<<<grid2(max_rb, count), 256, 0, s>>>(ddb, rows_b, nnz_b, brp);
    if (f32) {
      k_cat_entries<float><<<grid2(max_na, count), 256, 0, s>>>(dda, acl, reinterpret_cast<float *>(D(o_avl)));
      k_cat_entries<float><<<grid2(max_nb, count), 256, 0, s>>>(ddb, bcl, reinterpret_cast<float *>(D(o_bvl)));
    } else {
      k_cat_entries<double><<<grid2(max_na, count), 256, 0, s>>>(dda, acl, reinterpret_cast<double *>(D(o_avl)));
      k_cat_entries<double><<<grid2(max_nb, count), 256, 0, s>>>(ddb, bcl, reinterpret_cast<double *>(D(o_bvl)));
    }
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    g_last_cuda = (int)e;
    cudaGetLastError();
    scratch_free(ws, s);
    return NSPB_ERR_CUDA;
  }
  // the product of the block-diagonal operands, C_cat arrays allocated here
  nspb_csr_in Acat = {(int32_t)rows_a, (int32_t)rows_b, nnz_a, arp, acl, D(o_avl),
                      f32 ? NSPB_F32 : NSPB_F64, 0};
  nspb_csr_in Bcat = {(int32_t)rows_b, (int32_t)cols_b, nnz_b, brp, bcl, D(o_bvl),
                      f32 ? NSPB_F32 : NSPB_F64, 0};
  nspb_csr_out Ccat;
  std::memset(&Ccat, 0, sizeof(Ccat));
  Ccat.rowptr = crp;
  st = nspb_spgemm(&Acat, &Bcat, &Ccat, &o, stats);
  if (st) {
    cudaStreamSynchronize(s);
    scratch_free(ws, s);
    return st;
  }
  // per-product row pointers (one allocation) and columns shifted back
  int *rp_all = nullptr;
  st = alloc_out(reinterpret_cast<void **>(&rp_all), 4 * (size_t)(rows_a + count));
  if (!st) {
    // the largest product's C bounds the x extent (its rows and entries)
    const long long per = std::max<long long>(Ccat.nnz / std::max(count, 1) * 4, 1 << 16);
    k_split<<<grid2(per, count), 256, 0, s>>>(crp, d_ar, reinterpret_cast<const int *>(D(o_sh)),
                                               rp_all, Ccat.col);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      g_last_cuda = (int)e;
      st = NSPB_ERR_CUDA;
    }
  }
  // C_cat's row pointer is scratch: read each product's first entry back
  std::vector<int> crp_h(count + 1);
  if (!st) {
    int *starts = reinterpret_cast<int *>(D(o_st));
    k_gather_starts<<<grid_cap(count + 1), 256, 0, s>>>(crp, d_ar, count, starts);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(crp_h.data(), starts, 4 * (count + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
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
  for (int p = 0; p < count; ++p) {
    C[p].nrows = A[p].nrows;
    C[p].ncols = B[p].ncols;
    C[p].nnz = crp_h[p + 1] - crp_h[p];
    C[p].rowptr = rp_all + a_rows[p] + p;
    C[p].col = Ccat.col + crp_h[p];
    C[p].val = Ccat.val + crp_h[p];
    C[p].capacity = C[p].nnz;
  }
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
    } while (last < count && est + (double)A[last].nnz * (double)B[last].nnz /
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
