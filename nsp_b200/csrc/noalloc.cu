// nspb_spgemm_noalloc: the product with no memory allocation of any kind on
// the device or in pinned host memory.
//
// Who needs it: callers that must not call cudaMalloc (or any allocating
// routine) inside the product. A host framework that owns all device memory
// through its own pool and forbids allocations inside a call it dispatches,
// a real-time loop whose device memory is reserved up front, or a process
// running close to the HBM limit where a surprise allocation would fail.
// They pass C's arrays in, and the call's scratch (row counts, the bin
// permutation, counters and scan tile states) comes from one fixed array in
// device memory inside the library (reserved at the first call on each
// device, see below).
//
// The array is a file-scope __device__ variable of kNoAllocScratch bytes;
// every GPU that loads this library holds it until the process exits. A call
// needs 8 bytes per row of A plus a few KB (see Call::alloc_scratch), so A may
// have at most about 4.19 million rows (4,000,000 is always accepted); larger
// inputs are rejected with NSPB_ERR_CAPACITY and C->nnz = -1 before any GPU
// work starts (a C too small for nnz(C) gives NSPB_ERR_CAPACITY with C->nnz =
// the entries needed, so the two cases are told apart).
//
// All calls on a device share the one array and it keeps the previous
// call's contents: each call clears the counters and scan states it reads
// before use and overwrites the rest. Two calls whose GPU work overlaps (on
// different streams, or from different host threads) race on the array;
// serialise them.
//
// Device address: in host code the array's name is only a host-side stand-in
// for the symbol, not a device address. The first call on each device, with
// that device current, looks the address up with cudaGetSymbolAddress and
// keeps it; later calls reuse it. Make that first call before any stream
// capture begins.
//
// When the memory is taken: CUDA loads a library's device code lazily by
// default (CUDA_MODULE_LOADING=LAZY), module by module. The array lives in
// this file's module, which is loaded by that first symbol lookup, so the
// 32 MiB are reserved at the first call on a device, not when the library is
// loaded; the product kernels' modules likewise load at their first launch.
// A caller that must not see any allocation inside its working calls makes
// one warm-up call at set-up time: a tiny product (a few rows) reserves the
// array and loads every kernel the row-group path uses. (A zero-row call
// reserves the array only.) With CUDA_MODULE_LOADING=EAGER everything loads
// with the library.
//
// The cached address belongs to the device's primary context, which is
// assumed to live as long as the process: after cudaDeviceReset (or a
// released and recreated primary context) the cache is stale, so do not call
// this entry point again in such a process.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "spgemm_host.h"

namespace nspb {

constexpr size_t kNoAllocScratch = 32u << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratch];

// Device address of g_noalloc_scratch on the current device (nullptr on error).
static void *noalloc_scratch() {
  static std::mutex mu;
  static void *addr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      g_last_cuda = (int)e;
      cudaGetLastError();
      return nullptr;
    }
    addr[dev] = p;
  }
  return addr[dev];
}

}  // namespace nspb

using namespace nspb;

extern "C" int nspb_spgemm_noalloc(const nspb_csr_in *A, const nspb_csr_in *B,
                                   nspb_csr_out *C, const nspb_opts *opts,
                                   nspb_stats *stats) {
  if (!C || !C->rowptr || !C->col || !C->val || C->capacity < 0) return NSPB_ERR_INVALID;
  nspb_opts o;
  nspb_default_opts(&o);
  if (opts) o = *opts;
  if (o.precision != NSPB_PREC_FP64) return NSPB_ERR_UNSUPPORTED;
  o.timing = 0;  // events are resources this entry does not create
  Call call;
  call.allow_map = false;  // the entry maps would need memory of their own
  int st = call.init(A, B, &o);
  if (st) return st;
  if (call.scratch_bytes() > kNoAllocScratch) {  // more rows than the array serves
    C->nnz = -1;
    return NSPB_ERR_CAPACITY;
  }
  void *scratch = noalloc_scratch();
  if (!scratch) return NSPB_ERR_CUDA;
  call.ext_ws = static_cast<char *>(scratch);
  call.ext_bytes = kNoAllocScratch;
  HostStage stage;  // pageable: the two small reads are synchronous anyway
  std::memset(&stage, 0, sizeof(stage));
  call.stage = &stage;
  int64_t nnz = 0;
  st = call.symbolic(C->rowptr, &nnz);
  if (st) return st;
  if (nnz > C->capacity) {
    C->nnz = nnz;
    return NSPB_ERR_CAPACITY;
  }
  st = call.numeric(C->rowptr, C->col, C->val);
  if (!st) st = call.finish(stats);
  if (st) return st;
  C->nrows = A->nrows;
  C->ncols = B->ncols;
  C->nnz = nnz;
  return NSPB_OK;
}
