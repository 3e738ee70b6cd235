// C = A·B with A, B and C in host memory: the copies overlap the product.
//
// The reference's caller copies its matrices to the device, calls the product
// and copies C back, one step after the other (src/CSR.cu:656-683 copyToDevice
// / copyToHost around nsparseMGPU). Here, on three streams:
//   1. A's and B's row pointers and columns go to the device first on the
//      compute stream; their values follow on a value stream while the
//      symbolic phase runs (it needs no values);
//   2. C's row pointer comes back and cuts the rows into blocks of about
//      equal nnz;
//   3. each block's numeric step runs on the compute stream into one of two
//      device buffers, whose columns and values are copied to the caller's
//      host arrays on a third stream while the next block is computed.
// With pinned host arrays the D2H copy of C, the largest transfer, runs under
// the numeric phase. The values travel in row chunks, each with an event, and
// a row block's numeric step waits only for the chunks that hold its A rows
// and the B rows its columns reach (the largest column of each A chunk is
// found on the device before the symbolic phase). A banded product starts its
// numeric phase, and C's copy back, as soon as the symbolic phase ends, with
// most values still in flight the other way; a product whose rows reach every
// column waits for all of them.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "spgemm_host.h"

namespace nspb {

__global__ void k_rebase_slice(const int *__restrict__ in, int first, int n, int *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
    out[i] = in[first + i] - in[first];
}

// Value chunks of the host-operand product.
constexpr int kValChunks = 16;

__global__ void k_fold_err(const int *__restrict__ src, int *__restrict__ dst) {
  if (*src) atomicOr(dst, *src);
}

// colmax[j] = largest column of the A rows [j*chunk_rows, (j+1)*chunk_rows),
// -1 when they hold no entry (colmax starts at -1). A warp per row; the
// maxima of a block meet in shared memory first.
__global__ void __launch_bounds__(256)
    k_chunk_colmax(const int *__restrict__ arpt, const int *__restrict__ acol, int n,
                   int chunk_rows, int *__restrict__ colmax) {
  __shared__ int smax[kValChunks];
  if (threadIdx.x < kValChunks) smax[threadIdx.x] = -1;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int row = (blockIdx.x * 256 + (int)threadIdx.x) >> 5; row < n;
       row += (gridDim.x * 256) >> 5) {
    int m = -1;
    for (int j = arpt[row] + lane; j < arpt[row + 1]; j += 32) m = max(m, acol[j]);
    m = __reduce_max_sync(0xffffffffu, m);
    if (lane == 0 && m >= 0) atomicMax(&smax[row / chunk_rows], m);
  }
  __syncthreads();
  if (threadIdx.x < kValChunks && smax[threadIdx.x] >= 0)
    atomicMax(&colmax[threadIdx.x], smax[threadIdx.x]);
}

namespace {

struct Pool {
  cudaStream_t s;
  std::vector<void *> blocks;
  explicit Pool(cudaStream_t st) : s(st) {}
  ~Pool() {
    for (void *p : blocks) scratch_free(p, s);
  }
  template <typename T>
  int get(T **p, size_t count) {
    void *q = nullptr;
    const int st = scratch_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), s);
    if (st) return st;
    blocks.push_back(q);
    *p = static_cast<T *>(q);
    return NSPB_OK;
  }
};

struct Streams {
  cudaStream_t copy = nullptr;  // C device -> host
  cudaStream_t vals = nullptr;  // operand values host -> device
  cudaEvent_t ev[5 + kValChunks] = {};
  ~Streams() {
    drain();
    if (copy) cudaStreamDestroy(copy);
    if (vals) cudaStreamDestroy(vals);
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
  // waits for both copy streams; returns the first error
  cudaError_t drain() {
    const cudaError_t a = vals ? cudaStreamSynchronize(vals) : cudaSuccess;
    const cudaError_t b = copy ? cudaStreamSynchronize(copy) : cudaSuccess;
    return a != cudaSuccess ? a : b;
  }
};

int fail(cudaError_t e) {
  g_last_cuda = (int)e;
  cudaGetLastError();
  return NSPB_ERR_CUDA;
}

// Numeric step of one row block with no device-to-host read: a read queued
// behind the previous block's copy of C to the host would hold this block
// until that copy ends. The numeric bins come from C's row pointer on the host
// (rows of the block: c_rowptr[0..nrows]); the block's error word is folded
// into err on the device before its scratch is released.
int block_numeric(const nspb_csr_in *Ab, const nspb_csr_in *dB, nspb_csr_out *Cb,
                  const nspb_opts *ob, const int32_t *c_rowptr, int *err) {
  Call call;
  int st = call.init(Ab, dB, ob);
  if (st) return st;
  if ((st = call.alloc_scratch())) return st;
  for (int r = 0; r < Ab->nrows; ++r) {
    const int len = c_rowptr[r + 1] - c_rowptr[r];
    if (len > 0) ++call.h.num_counts[num_bin_of(len, call.lim)];
  }
  call.b_sorted = ob->assume_sorted != 0;
  call.num_counts_ready = true;
  call.h.total_nnz = Cb->nnz;
  if ((st = call.numeric(Cb->rowptr, Cb->col, Cb->val))) return st;
  k_fold_err<<<1, 1, 0, call.s>>>(&call.ctr->err, err);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? NSPB_OK : fail(e);
}

bool valid_host(const nspb_csr_in *M) {
  if (!M || M->nrows < 0 || M->ncols < 0 || M->nnz < 0 || M->nnz > INT32_MAX) return false;
  if (!M->rowptr) return false;
  if (M->nnz > 0 && (!M->col || !M->val)) return false;
  return M->val_type == NSPB_F64 || M->val_type == NSPB_F32;
}

}  // namespace
}  // namespace nspb

using namespace nspb;

extern "C" int nspb_spgemm_host(const nspb_csr_in *hA, const nspb_csr_in *hB, int32_t *h_rowptr,
                                int32_t *h_col, double *h_val, int64_t h_capacity,
                                int64_t *nnz_out, int32_t nblocks, const nspb_opts *opts) {
  if (!valid_host(hA) || !valid_host(hB) || !h_rowptr || !nnz_out) return NSPB_ERR_INVALID;
  if (hA->ncols != hB->nrows || hA->val_type != hB->val_type) return NSPB_ERR_INVALID;
  if (hA->rowptr[0] != 0 || hB->rowptr[0] != 0 || hA->rowptr[hA->nrows] != hA->nnz ||
      hB->rowptr[hB->nrows] != hB->nnz)
    return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  o.timing = 0;
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NSPB_ERR_NO_DEVICE;
  }
  const size_t vsz = hA->val_type == NSPB_F32 ? 4 : 8;
  const bool same = hA->rowptr == hB->rowptr && hA->col == hB->col && hA->val == hB->val &&
                    hA->nrows == hB->nrows && hA->nnz == hB->nnz;
  const int n = hA->nrows;
  Streams ss;
  cudaError_t e = cudaStreamCreateWithFlags(&ss.copy, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ss.vals, cudaStreamNonBlocking);
  for (int i = 0; i < 5 + kValChunks && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&ss.ev[i], cudaEventDisableTiming);
  if (e != cudaSuccess) return fail(e);
  cudaEvent_t &ev_alloc = ss.ev[0];
  cudaEvent_t *computed = ss.ev + 1, *copied = ss.ev + 3, *chunk_done = ss.ev + 5;
  // value chunks: A rows [j*ca, (j+1)*ca) and B rows [j*cb, (j+1)*cb)
  const int ca = (int)std::max<int64_t>(1, ((int64_t)n + kValChunks - 1) / kValChunks);
  const int cb = (int)std::max<int64_t>(1, ((int64_t)hB->nrows + kValChunks - 1) / kValChunks);
  Pool pool(s);
  int st;
  // 1. device operands: structure on the compute stream, values on the copy stream
  int *arp = nullptr, *acl = nullptr, *brp = nullptr, *bcl = nullptr;
  char *aval = nullptr, *bval = nullptr;
  if ((st = pool.get(&arp, (size_t)n + 1)) || (st = pool.get(&acl, (size_t)hA->nnz)) ||
      (st = pool.get(&aval, (size_t)hA->nnz * vsz)))
    return st;
  if (same) {
    brp = arp;
    bcl = acl;
    bval = aval;
  } else if ((st = pool.get(&brp, (size_t)hB->nrows + 1)) ||
             (st = pool.get(&bcl, (size_t)hB->nnz)) ||
             (st = pool.get(&bval, (size_t)hB->nnz * vsz))) {
    return st;
  }
  auto h2d = [&](void *d, const void *h, size_t bytes, cudaStream_t st_) {
    return bytes ? cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st_) : cudaSuccess;
  };
  e = h2d(arp, hA->rowptr, ((size_t)n + 1) * 4, s);
  if (e == cudaSuccess) e = h2d(acl, hA->col, (size_t)hA->nnz * 4, s);
  if (e == cudaSuccess && !same) e = h2d(brp, hB->rowptr, ((size_t)hB->nrows + 1) * 4, s);
  if (e == cudaSuccess && !same) e = h2d(bcl, hB->col, (size_t)hB->nnz * 4, s);
  if (e == cudaSuccess) e = cudaEventRecord(ev_alloc, s);  // allocations ordered first
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ss.vals, ev_alloc, 0);
  auto val_rows = [&](const nspb_csr_in *H, char *d, int64_t r0_, int64_t r1_) {
    const int r0 = (int)std::min<int64_t>(r0_, H->nrows), r1 = (int)std::min<int64_t>(r1_, H->nrows);
    if (r0 >= r1) return cudaSuccess;
    const size_t b0 = (size_t)H->rowptr[r0] * vsz, b1 = (size_t)H->rowptr[r1] * vsz;
    return h2d(d + b0, static_cast<const char *>(H->val) + b0, b1 - b0, ss.vals);
  };
  for (int j = 0; j < kValChunks && e == cudaSuccess; ++j) {
    e = val_rows(hA, aval, (int64_t)j * ca, (int64_t)(j + 1) * ca);
    if (e == cudaSuccess && !same) e = val_rows(hB, bval, (int64_t)j * cb, (int64_t)(j + 1) * cb);
    if (e == cudaSuccess) e = cudaEventRecord(chunk_done[j], ss.vals);
  }
  if (e != cudaSuccess) {
    ss.drain();
    return fail(e);
  }
  const nspb_csr_in dA = {n, hA->ncols, hA->nnz, arp, acl, aval, hA->val_type, 0};
  const nspb_csr_in dB = {hB->nrows, hB->ncols, hB->nnz, brp, bcl, bval, hB->val_type, 0};
  // 2. largest column per A chunk, symbolic phase (no values needed), C's row
  // pointer to the host
  int *crpt = nullptr, *colmax = nullptr;  // colmax[kValChunks]: then the error word
  if ((st = pool.get(&crpt, (size_t)n + 1)) || (st = pool.get(&colmax, kValChunks + 1))) {
    ss.drain();
    return st;
  }
  int *d_err = colmax + kValChunks;
  e = cudaMemsetAsync(colmax, 0xff, kValChunks * sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
  if (e == cudaSuccess && n > 0) {
    const int grid = (int)std::min<int64_t>(((int64_t)n * 32 + 255) / 256, dev_info().sms * 8);
    k_chunk_colmax<<<grid, 256, 0, s>>>(arp, acl, n, ca, colmax);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    ss.drain();
    return fail(e);
  }
  int h_colmax[kValChunks];
  int64_t nnz = 0;
  bool b_sorted = true;
  {
    Call sym;
    sym.allow_map = false;  // the row blocks' numeric steps run in their own calls
    if (!(st = sym.init(&dA, &dB, &o))) st = sym.symbolic(crpt, &nnz);
    b_sorted = sym.b_sorted;
  }
  if (!st) {
    e = cudaMemcpyAsync(h_rowptr, crpt, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_colmax, colmax, sizeof(h_colmax), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = fail(e);
  }
  if (st) {
    ss.drain();
    return st;
  }
  *nnz_out = nnz;
  if (!h_col || !h_val || h_capacity < nnz) {
    ss.drain();
    return nnz == 0 ? NSPB_OK : NSPB_ERR_CAPACITY;
  }
  // 3. row blocks of about nnz/nb entries, two buffers in flight
  // 16 blocks by default: the copy of C back starts after the first block, so
  // a smaller first block starts it sooner (27-pt 128^3: 66.1 -> 65.5 ms)
  const int nb = std::max(1, std::min(nblocks > 0 ? nblocks : 16, std::max(n, 1)));
  std::vector<int> cut(1, 0);
  for (int k = 1; k < nb; ++k) {
    const long long target = nnz * k / nb;
    const int r = (int)(std::lower_bound(h_rowptr, h_rowptr + n + 1, (int32_t)target) - h_rowptr);
    if (r > cut.back() && r < n) cut.push_back(r);
  }
  cut.push_back(n);
  long long max_rows = 0, max_nnz = 0;
  for (size_t k = 0; k + 1 < cut.size(); ++k) {
    max_rows = std::max<long long>(max_rows, cut[k + 1] - cut[k]);
    max_nnz = std::max<long long>(max_nnz, (long long)h_rowptr[cut[k + 1]] - h_rowptr[cut[k]]);
  }
  int *bcrp[2] = {nullptr, nullptr}, *bcol[2] = {nullptr, nullptr};
  double *bvl[2] = {nullptr, nullptr};
  for (int b = 0; b < 2 && !st; ++b)
    if ((st = pool.get(&bcrp[b], (size_t)max_rows + 1)) || (st = pool.get(&bcol[b], (size_t)max_nnz)) ||
        (st = pool.get(&bvl[b], (size_t)max_nnz)))
      break;
  nspb_opts ob = o;
  ob.assume_sorted = b_sorted ? 1 : 0;  // checked once by the symbolic phase
  for (size_t k = 0; k + 1 < cut.size() && !st; ++k) {
    const int b = (int)(k & 1);
    const int r0 = cut[k], r1 = cut[k + 1], nr = r1 - r0;
    const long long c0 = h_rowptr[r0], cnt = (long long)h_rowptr[r1] - c0;
    if (k >= 2 && (e = cudaStreamWaitEvent(s, copied[b], 0)) != cudaSuccess) {
      st = fail(e);
      break;
    }
    // the value chunks holding rows [r0, r1) of A and every B row they reach
    int need = std::max(r1 - 1, 0) / ca, reach = -1;
    for (int j = r0 / ca; j <= need; ++j) reach = std::max(reach, h_colmax[j]);
    if (reach >= 0) need = std::max(need, std::min(reach, hB->nrows - 1) / cb);
    if ((e = cudaStreamWaitEvent(s, chunk_done[std::min(need, kValChunks - 1)], 0)) !=
        cudaSuccess) {
      st = fail(e);
      break;
    }
    k_rebase_slice<<<std::max(1, std::min((nr + 256) / 256, dev_info().sms * 8)), 256, 0, s>>>(
        crpt, r0, nr, bcrp[b]);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      st = fail(e);
      break;
    }
    const nspb_csr_in Ab = {nr, hA->ncols, (int64_t)hA->rowptr[r1] - hA->rowptr[r0], arp + r0, acl,
                            aval, hA->val_type, 0};
    nspb_csr_out Cb = {nr, hB->ncols, cnt, bcrp[b], bcol[b], bvl[b], max_nnz};
    if ((st = block_numeric(&Ab, &dB, &Cb, &ob, h_rowptr + r0, d_err))) break;
    e = cudaEventRecord(computed[b], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ss.copy, computed[b], 0);
    if (e == cudaSuccess && cnt > 0)
      e = cudaMemcpyAsync(h_col + c0, bcol[b], (size_t)cnt * 4, cudaMemcpyDeviceToHost, ss.copy);
    if (e == cudaSuccess && cnt > 0)
      e = cudaMemcpyAsync(h_val + c0, bvl[b], (size_t)cnt * 8, cudaMemcpyDeviceToHost, ss.copy);
    if (e == cudaSuccess) e = cudaEventRecord(copied[b], ss.copy);
    if (e != cudaSuccess) st = fail(e);
  }
  e = ss.drain();
  if (!st && e != cudaSuccess) st = fail(e);
  int h_err = 0;
  e = cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (!st && e != cudaSuccess) st = fail(e);
  if (!st && h_err) st = NSPB_ERR_DEVICE;
  return st;
}
