// Device memory arena: the request loop's contexts take their buffers from
// it instead of cudaMalloc.
//
// A served context lives for one request or a few; creating one costs about
// forty cudaMalloc calls and returning it to the driver as many cudaFree
// calls, and each of those may wait on the driver's page-table work for
// gigabytes. The arena claims HBM in large blocks (cudaMalloc once per
// block, kept until the arena is destroyed) and hands out sub-ranges through
// a RangePool (arena_core.h): best fit over the free ranges, a released
// range merged with its free neighbours inside the same block, ranges of
// whole 256-byte units at 256-byte-aligned addresses like cudaMalloc's, which
// the tensor maps (16-byte base) and vector loads rely on. When no free range
// fits, a new block of max(request, growth step) is claimed from the driver.
// The arena knows nothing of streams: a range must not be released while
// queued work may still touch it. Contexts synchronise their own streams
// before they release buffers (quiesce in engine.cu). All calls are
// thread-safe.
#include <mutex>

#include "arena_core.h"
#include "engine_internal.cuh"

namespace tpm {

struct DeviceArena {
  int device = 0;
  int64_t step = 1ll << 30;  // growth block size
  std::mutex mu;
  RangePool pool;
};

namespace {

// Claims a new block of at least n bytes from the driver (a->mu held).
cudaError_t grow(DeviceArena *a, size_t n) {
  size_t bytes = RangePool::round(n > (size_t)a->step ? n : (size_t)a->step);
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e;
  }
  a->pool.add_block((char *)p, bytes);
  return cudaSuccess;
}

}  // namespace

DeviceArena *arena_create(int device, int64_t step_bytes) {
  DeviceArena *a = new DeviceArena();
  a->device = device;
  if (step_bytes > 0) a->step = step_bytes;
  return a;
}

void arena_destroy(DeviceArena *a) {
  if (!a) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(a->device);
  for (auto &b : a->pool.blocks()) cudaFree(b.first);
  cudaSetDevice(prev);
  delete a;
}

cudaError_t arena_reserve(DeviceArena *a, int64_t bytes) {
  std::lock_guard<std::mutex> lk(a->mu);
  int64_t free_bytes = a->pool.reserved() - a->pool.in_use();
  if (bytes <= free_bytes) return cudaSuccess;
  return grow(a, (size_t)(bytes - free_bytes));
}

void arena_usage(DeviceArena *a, int64_t *reserved, int64_t *in_use) {
  std::lock_guard<std::mutex> lk(a->mu);
  if (reserved) *reserved = a->pool.reserved();
  if (in_use) *in_use = a->pool.in_use();
}

cudaError_t arena_alloc(DeviceArena *a, void **out, size_t bytes) {
  std::lock_guard<std::mutex> lk(a->mu);
  char *p = a->pool.alloc(bytes);
  if (!p) {
    cudaError_t e = grow(a, RangePool::round(bytes));
    if (e != cudaSuccess) {
      *out = nullptr;
      return e;
    }
    p = a->pool.alloc(bytes);
  }
  *out = p;
  return p ? cudaSuccess : cudaErrorMemoryAllocation;
}

void arena_free(DeviceArena *a, void *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(a->mu);
  a->pool.release((char *)p);
}

cudaError_t dmalloc(DeviceArena *a, void **p, size_t bytes) {
  if (a) return arena_alloc(a, p, bytes);
  return cudaMalloc(p, bytes);
}

void dfree(DeviceArena *a, void *p) {
  if (!p) return;
  if (a)
    arena_free(a, p);
  else
    cudaFree(p);
}

}  // namespace tpm
