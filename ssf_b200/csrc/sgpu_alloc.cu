// The device-block cache behind DevBuf.
//
// Handles own large device arrays (the CSR and 3x3-block copies of a
// 1M-equation matrix are about 1.5 GB); building and destroying one per solve
// paid cudaMalloc and cudaFree for each, about 10 ms on B200 for the destroy
// alone.  Released blocks are kept here, per device, and handed out again for
// requests that fit them without wasting more than half; a request that
// cudaMalloc cannot meet returns the cached blocks to the driver first.
//
// Ordering: cudaFree waits for the device's outstanding work, and code that
// releases a buffer may rely on that; devmem_put keeps the guarantee with a
// cudaDeviceSynchronize before the block becomes reusable.  Contents: memory
// fresh from cudaMalloc reads as zeros in practice and device flags and
// counters of this library start from that, so a reused block is cleared
// (and the clear finished) before it is handed out.
#include <map>
#include <mutex>

#include "sgpu_internal.cuh"

namespace sgpu {
namespace {

struct Block {
  void *p;
  int dev;
};

std::mutex g_mu;
std::multimap<size_t, Block> g_free;  // bytes -> block
size_t g_cached = 0;
constexpr size_t kCacheCap = size_t(24) << 30;  // bytes kept idle at most

size_t round_bytes(size_t b) {
  if (b <= (size_t(1) << 20)) {  // small: powers of two from 512 B
    size_t r = 512;
    while (r < b) r <<= 1;
    return r;
  }
  const size_t g = size_t(2) << 20;  // large: 2 MiB granules
  return (b + g - 1) / g * g;
}

void flush_locked(int dev) {
  for (auto it = g_free.begin(); it != g_free.end();) {
    if (dev < 0 || it->second.dev == dev) {
      int cur = 0;
      cudaGetDevice(&cur);
      if (it->second.dev != cur) cudaSetDevice(it->second.dev);
      cudaFree(it->second.p);
      if (it->second.dev != cur) cudaSetDevice(cur);
      g_cached -= it->first;
      it = g_free.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace

cudaError_t devmem_get(void **p, size_t *bytes) {
  const size_t want = round_bytes(*bytes);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_free.lower_bound(want); it != g_free.end() && it->first <= 2 * want; ++it) {
      if (it->second.dev != dev) continue;
      *p = it->second.p;
      *bytes = it->first;
      g_cached -= it->first;
      g_free.erase(it);
      cudaError_t z = cudaMemset(*p, 0, *bytes);
      if (z == cudaSuccess) z = cudaDeviceSynchronize();
      return z;
    }
  }
  e = cudaMalloc(p, want);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    std::lock_guard<std::mutex> lk(g_mu);
    flush_locked(dev);
    e = cudaMalloc(p, want);
  }
  if (e == cudaSuccess) *bytes = want;
  return e;
}

void devmem_put(void *p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceSynchronize() != cudaSuccess) {  // a failed context: give the block back
    cudaFree(p);
    return;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_free.emplace(bytes, Block{p, dev});
  g_cached += bytes;
  while (g_cached > kCacheCap && !g_free.empty()) {  // drop the largest idle blocks
    auto it = std::prev(g_free.end());
    cudaFree(it->second.p);
    g_cached -= it->first;
    g_free.erase(it);
  }
}

}  // namespace sgpu
