// Process-wide cache of device and pinned host blocks (devmem.h).
#include "devmem.h"

#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace dmm {
namespace {

// Size class: powers of two up to 1 MiB, then multiples of 2 MiB.
size_t size_class(size_t b) {
  if (b <= 512) return 512;
  if (b <= (size_t(1) << 20)) {
    size_t c = 512;
    while (c < b) c <<= 1;
    return c;
  }
  const size_t g = size_t(2) << 20;
  return (b + g - 1) / g * g;
}

struct Block {
  int dev;  // -1: pinned host memory
  size_t bytes;
};

struct Cache {
  std::mutex mu;
  std::unordered_map<void*, Block> live;             // handed out
  std::map<std::pair<int, size_t>, std::vector<void*>> idle;  // (dev, class) -> blocks
  std::unordered_map<int, size_t> idle_bytes;        // per dev
};

Cache& cache() {
  static Cache* c = new Cache();  // never destroyed: blocks may be freed at exit
  return *c;
}

cudaError_t take(void** p, size_t bytes, int dev) {
  const size_t cls = size_class(bytes == 0 ? 1 : bytes);
  Cache& c = cache();
  {
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.idle.find({dev, cls});
    if (it != c.idle.end() && !it->second.empty()) {
      *p = it->second.back();
      it->second.pop_back();
      c.idle_bytes[dev] -= cls;
      c.live[*p] = Block{dev, cls};
      return cudaSuccess;
    }
  }
  void* q = nullptr;
  cudaError_t e = dev >= 0 ? cudaMalloc(&q, cls) : cudaMallocHost(&q, cls);
  if (e != cudaSuccess) {
    cudaGetLastError();
    // the cache may hold the memory this request needs: give it back and retry once
    release_cached();
    e = dev >= 0 ? cudaMalloc(&q, cls) : cudaMallocHost(&q, cls);
    if (e != cudaSuccess) return e;
  }
  std::lock_guard<std::mutex> g(c.mu);
  c.live[q] = Block{dev, cls};
  *p = q;
  return cudaSuccess;
}

void give(void* p) {
  if (!p) return;
  Cache& c = cache();
  Block b;
  {
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) return;
    b = it->second;
    c.live.erase(it);
    if (c.idle_bytes[b.dev] + b.bytes <= kDevCacheBytes) {
      c.idle[{b.dev, b.bytes}].push_back(p);
      c.idle_bytes[b.dev] += b.bytes;
      return;
    }
  }
  if (b.dev >= 0) {
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(b.dev);
    cudaFree(p);
    if (cur >= 0) cudaSetDevice(cur);
  } else {
    cudaFreeHost(p);
  }
}

}  // namespace

cudaError_t dev_alloc_raw(void** p, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  return take(p, bytes, dev);
}

void dev_free(void* p) { give(p); }

cudaError_t pinned_alloc_raw(void** p, size_t bytes) { return take(p, bytes, -1); }

void pinned_free(void* p) { give(p); }

void release_cached() {
  Cache& c = cache();
  std::map<std::pair<int, size_t>, std::vector<void*>> idle;
  {
    std::lock_guard<std::mutex> g(c.mu);
    idle.swap(c.idle);
    c.idle_bytes.clear();
  }
  int cur = -1;
  cudaGetDevice(&cur);
  for (auto& kv : idle) {
    const int dev = kv.first.first;
    if (dev >= 0) cudaSetDevice(dev);
    for (void* p : kv.second) {
      if (dev >= 0) cudaFree(p);
      else cudaFreeHost(p);
    }
  }
  if (cur >= 0) cudaSetDevice(cur);
}

}  // namespace dmm
