// pool.cu -- caching device allocator of the engine.
//
// The engine, the list store and the split operands allocate and release
// tens of buffers per CC solve (up to tens of GB).  cudaMalloc/cudaFree of
// that much memory costs milliseconds to seconds per solve (the driver maps
// and unmaps pages, cudaFree synchronises the device), which dominates short
// solves such as the 64-system batch.  Released blocks are therefore kept per
// device and size class and handed out again; they return to the driver only
// when an allocation would otherwise fail, or at aces_fin.
#include <atomic>
#include <map>
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace acesb200 {

namespace {
struct Pool {
  std::mutex mu;
  std::multimap<std::pair<int, size_t>, void *> free_blocks;   // (device, bytes) -> block
  std::unordered_map<void *, std::pair<int, size_t>> live;     // block -> (device, bytes)
  std::map<int, size_t> cached;                                // device -> cached bytes
  std::map<int, size_t> cap;                                   // device -> cache limit
};
// cached bytes per device are held below 35 % of its memory, so other users of
// the device in the same process (e.g. a host program's own allocator) keep room
size_t cache_cap(Pool &P, int dev) {
  auto it = P.cap.find(dev);
  if (it != P.cap.end()) return it->second;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    tot = 0;
  }
  const size_t c = tot / 100 * 35;
  P.cap[dev] = c;
  return c;
}
// every dev_alloc call, and the ones the cache could not serve (cudaMalloc)
std::atomic<long long> g_alloc_calls{0}, g_driver_allocs{0};
Pool &pool() {
  static Pool *p = new Pool();  // never destroyed: blocks may be released at exit
  return *p;
}
size_t size_class(size_t bytes) {
  if (bytes == 0) bytes = 1;
  if (bytes >= (2u << 20)) return (bytes + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
  size_t c = 512;
  while (c < bytes) c <<= 1;
  return c;
}
void trim_device(Pool &P, int dev) {
  for (auto it = P.free_blocks.begin(); it != P.free_blocks.end();) {
    if (it->first.first == dev) {
      cudaFree(it->second);
      it = P.free_blocks.erase(it);
    } else {
      ++it;
    }
  }
  P.cached[dev] = 0;
}
}  // namespace

cudaError_t dev_alloc(void **ptr, size_t bytes) {
  *ptr = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const size_t cls = size_class(bytes);
  g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
  Pool &P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  // smallest cached block of this device that fits without wasting more than
  // a quarter of it
  auto it = P.free_blocks.lower_bound({dev, cls});
  if (it != P.free_blocks.end() && it->first.first == dev &&
      it->first.second <= cls + cls / 4) {
    *ptr = it->second;
    P.live[*ptr] = it->first;
    P.cached[dev] -= it->first.second;
    P.free_blocks.erase(it);
    return cudaSuccess;
  }
  g_driver_allocs.fetch_add(1, std::memory_order_relaxed);
  e = cudaMalloc(ptr, cls);
  if (e != cudaSuccess) {
    cudaGetLastError();
    trim_device(P, dev);
    e = cudaMalloc(ptr, cls);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *ptr = nullptr;
      return e;
    }
  }
  P.live[*ptr] = {dev, cls};
  return cudaSuccess;
}

void dev_free(void *ptr) {
  if (!ptr) return;
  Pool &P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.live.find(ptr);
  if (it == P.live.end()) return;  // not ours
  const int dev = it->second.first;
  const size_t bytes = it->second.second;
  P.live.erase(it);
  int cur = -1;
  cudaGetDevice(&cur);
  const size_t cap = cur == dev ? cache_cap(P, dev) : 0;
  if (P.cached[dev] + bytes > cap) {
    // over the limit: release cached blocks of this device, largest first,
    // then the block itself if it still does not fit
    while (P.cached[dev] + bytes > cap) {
      auto last = P.free_blocks.lower_bound({dev + 1, 0});
      if (last == P.free_blocks.begin()) break;
      --last;
      if (last->first.first != dev) break;
      cudaFree(last->second);
      P.cached[dev] -= last->first.second;
      P.free_blocks.erase(last);
    }
    if (P.cached[dev] + bytes > cap) {
      cudaFree(ptr);
      return;
    }
  }
  P.free_blocks.emplace(std::make_pair(dev, bytes), ptr);
  P.cached[dev] += bytes;
}

void pool_trim() {
  Pool &P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  for (auto &kv : P.free_blocks) cudaFree(kv.second);
  P.free_blocks.clear();
  P.cached.clear();
}

}  // namespace acesb200

extern "C" int aces_pool_stats(long long *alloc_calls, long long *driver_allocs,
                               long long *cached_bytes) {
  using namespace acesb200;
  if (alloc_calls) *alloc_calls = g_alloc_calls.load();
  if (driver_allocs) *driver_allocs = g_driver_allocs.load();
  if (cached_bytes) {
    Pool &P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    long long c = 0;
    for (auto &kv : P.cached) c += (long long)kv.second;
    *cached_bytes = c;
  }
  return ACES_OK;
}
