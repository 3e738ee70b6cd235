// Host helpers for launching persistent grids: per-device opt-in shared
// memory and occupancy, cached per (device, kernel, block, smem).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "internal.h"

namespace nspb {

// Resident CTAs per SM for `func` at (threads, smem); sets the opt-in
// dynamic shared memory limit first when smem > 48 KB. Returns 0 on error.
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
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return 0;
  }
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

}  // namespace nspb
