// Device and pinned host memory of packs, through a process-wide cache.
//
// cudaMalloc and cudaFree cost 0.1-1 ms each and cudaFree synchronizes the device, so an
// instance that is created, stepped a few dozen times and destroyed would spend most of its
// time in the driver's allocator.  Blocks freed here go to a per-device cache (keyed by the
// rounded size) and are handed to the next request of the same size class; the cache keeps
// at most kDevCacheBytes per device (beyond that, blocks go back to the driver), and
// release_cached() returns everything.  A block must be idle on the GPU when it is freed:
// the caller synchronizes its stream first.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace dmm {

constexpr size_t kDevCacheBytes = size_t(8) << 30;

cudaError_t dev_alloc_raw(void** p, size_t bytes);  // on the current device
void dev_free(void* p);
cudaError_t pinned_alloc_raw(void** p, size_t bytes);
void pinned_free(void* p);
void release_cached();  // all devices' cached blocks and cached pinned blocks

template <class T>
inline cudaError_t dev_alloc(T** p, size_t bytes) {
  return dev_alloc_raw(reinterpret_cast<void**>(p), bytes);
}
template <class T>
inline cudaError_t pinned_alloc(T** p, size_t bytes) {
  return pinned_alloc_raw(reinterpret_cast<void**>(p), bytes);
}

}  // namespace dmm
