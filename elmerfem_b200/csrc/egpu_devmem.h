// egpu_devmem.h -- device memory blocks for the library's buffers (host-only header).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdlib>
#include <iterator>
#include <map>
#include <mutex>

namespace egpu {

// device memory: a per-device cache of freed blocks
//
// Requests of the serving engine and the batched solver clone, fill and free a matrix's
// device objects (twenty-odd buffers) per request.  cudaMalloc / cudaFree of large blocks
// cost milliseconds each and vary with the driver's state (measured on B200: 1 to 5 s of
// allocation and free per 48-request serving stream, varying from run to run).  Freed blocks therefore
// stay in a process-wide cache, by device, and are handed out again to requests of a size
// between two thirds of the block's size and its full size.  A release first synchronises the device,
// as cudaFree does implicitly, so no queued kernel can still use a block when it is reused.
// At most devcache_max() bytes are kept.  An allocation that fails gives cached blocks back to
// the driver, largest first, until the freed bytes cover the request, and retries; only when
// that is not enough does it empty the device's cache.  (Emptying it on every failure cost
// seconds of cudaFree per serving stream once the cache was large.)
constexpr size_t DEVCACHE_GRAIN = (size_t)1 << 16;   // blocks are multiples of 64 KB

// bytes kept in the cache per device: 24 GB, or EGPU_DEVCACHE_GB
inline size_t devcache_max() {
  static const size_t v = [] {
    const char *e = std::getenv("EGPU_DEVCACHE_GB");
    const double gb = e ? std::atof(e) : 24.0;
    return (size_t)((gb > 0 ? gb : 0.0) * (double)(1ull << 30));
  }();
  return v;
}

struct DevCache {
  std::mutex mu;
  std::map<int, std::multimap<size_t, void *>> free_blocks;  // device -> size -> block
  std::map<int, size_t> cached;                                 // device -> bytes held
};
inline DevCache &devcache() {
  static DevCache *c = new DevCache;  // never destroyed: blocks go back with the process
  return *c;
}
inline size_t devcache_round(size_t bytes) { return (bytes + DEVCACHE_GRAIN - 1) / DEVCACHE_GRAIN * DEVCACHE_GRAIN; }

// a block of at least `bytes` on the current device; *cap receives its size
inline cudaError_t dev_alloc(void **p, size_t bytes, size_t *cap, int *dev) {
  cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) return e;
  const size_t want = devcache_round(bytes);
  DevCache &c = devcache();
  {
    std::lock_guard<std::mutex> g(c.mu);
    auto &fb = c.free_blocks[*dev];
    auto it = fb.lower_bound(want);
    if (it != fb.end() && it->first <= want + want / 2) {
      *p = it->second;
      *cap = it->first;
      c.cached[*dev] -= it->first;
      fb.erase(it);
      return cudaSuccess;
    }
  }
  e = cudaMalloc(p, want);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the non-sticky allocation error before retrying
    std::lock_guard<std::mutex> g(c.mu);
    auto &fb = c.free_blocks[*dev];
    // largest blocks first, until the bytes given back cover the request; then everything
    size_t given = 0;
    while (!fb.empty() && given < want) {
      auto last = std::prev(fb.end());
      cudaFree(last->second);
      given += last->first;
      c.cached[*dev] -= last->first;
      fb.erase(last);
    }
    e = cudaMalloc(p, want);
    if (e == cudaErrorMemoryAllocation && !fb.empty()) {
      cudaGetLastError();
      for (auto &kv : fb) cudaFree(kv.second);
      fb.clear();
      c.cached[*dev] = 0;
      e = cudaMalloc(p, want);
    }
  }
  if (e == cudaSuccess) *cap = want;
  return e;
}

// return a block (allocated on device dev) to the cache, or to the driver past the cap
inline void dev_free(void *p, size_t cap, int dev) {
  if (!p) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  cudaDeviceSynchronize();
  DevCache &c = devcache();
  bool keep = false;
  {
    std::lock_guard<std::mutex> g(c.mu);
    if (c.cached[dev] + cap <= devcache_max()) {
      c.free_blocks[dev].emplace(cap, p);
      c.cached[dev] += cap;
      keep = true;
    }
  }
  if (!keep) cudaFree(p);
  if (cur != dev && cur >= 0) cudaSetDevice(cur);
}

// bytes held in the cache for device dev (every device if dev < 0)
inline long long devcache_bytes(int dev) {
  DevCache &c = devcache();
  std::lock_guard<std::mutex> g(c.mu);
  long long t = 0;
  for (auto &kv : c.cached)
    if (dev < 0 || kv.first == dev) t += (long long)kv.second;
  return t;
}

// give the cached blocks of device dev (every device if dev < 0) back to the driver
inline long long devcache_release(int dev) {
  DevCache &c = devcache();
  std::lock_guard<std::mutex> g(c.mu);
  long long t = 0;
  bool any = false;
  for (auto &kv : c.free_blocks) any = any || ((dev < 0 || kv.first == dev) && !kv.second.empty());
  if (!any) return 0;
  int cur = -1;
  cudaGetDevice(&cur);
  for (auto &kv : c.free_blocks) {
    if (dev >= 0 && kv.first != dev) continue;
    if (kv.second.empty()) continue;
    cudaSetDevice(kv.first);
    cudaDeviceSynchronize();
    for (auto &b : kv.second) {
      cudaFree(b.second);
      t += (long long)b.first;
    }
    kv.second.clear();
    c.cached[kv.first] = 0;
  }
  if (cur >= 0) cudaSetDevice(cur);
  return t;
}

}  // namespace egpu
