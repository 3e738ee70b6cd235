// Host helpers for launching persistent grids: per-device opt-in shared
// memory and occupancy, cached per (device, kernel, block, smem).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "internal.h"

namespace nspb {

// Raises the dynamic shared memory limit of `func` to what the device allows
// beside its static shared memory, once per (device, kernel): launches of one
// kernel may then use any size up to that (a kernel whose static and dynamic
// parts add up past 48 KB needs the opt-in even when the dynamic part alone
// does not). Returns false on error.
inline bool allow_smem(const void *func) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, bool> done;
  const int dev = dev_info().device;
  const auto key = std::make_pair(dev, func);
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find(key);
  if (it != done.end()) return it->second;
  cudaFuncAttributes fa;
  bool ok = cudaFuncGetAttributes(&fa, func) == cudaSuccess;
  if (ok) {
    const int dyn = dev_info().smem_optin - (int)fa.sharedSizeBytes;
    ok = dyn > 0 &&
         cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) ==
             cudaSuccess;
  }
  if (!ok) cudaGetLastError();
  done[key] = ok;
  return ok;
}

// Resident CTAs per SM for `func` at (threads, smem), after raising its
// dynamic shared memory limit. Returns 0 on error.
inline int resident_ctas(const void *func, int threads, int smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void *, int, int>, int> cache;
  const int dev = dev_info().device;
  const auto key = std::make_tuple(dev, func, threads, smem);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  if (!allow_smem(func)) return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, func, threads, (size_t)smem) != cudaSuccess)
    return 0;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = blocks;
  return blocks;
}

// Grid for a grid-stride loop over `items` work items of `per_cta` each:
// no more CTAs than can be resident at once.
inline int persistent_grid(const void *func, int threads, int smem, long long items,
                           int per_cta) {
  const int occ = resident_ctas(func, threads, smem);
  if (occ <= 0) return 0;
  const long long need = (items + per_cta - 1) / per_cta;
  const long long cap = (long long)occ * dev_info().sms;
  return (int)(need < cap ? need : cap);
}

// Rows a row group takes in a run (row templates), at most `run`: a bin too
// small to give every resident group `run` rows gets shorter runs (1: no
// templates), so that its rows still spread over all the groups instead of
// queueing behind a few. A negative run is the caller's own (-run rows, as
// given).
inline int template_chunk(int run, long long count, const void *func, int threads, int smem,
                          int per_cta) {
  if (run < 0) return -run;
  if (run <= 1) return 1;
  const int occ = resident_ctas(func, threads, smem);
  const long long groups = (long long)(occ > 0 ? occ : 1) * dev_info().sms * per_cta;
  const long long fit = count / groups;
  return (int)(fit < run ? (fit > 1 ? fit : 1) : run);
}

}  // namespace nspb
