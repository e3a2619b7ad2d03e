// Device memory arena: the request loop's contexts take their buffers from
// it instead of cudaMalloc.
//
// A served context lives for one request or a few; creating one costs about
// forty cudaMalloc calls and returning it to the driver as many cudaFree
// calls, and each of those may wait on the driver's page-table work for
// gigabytes. The arena claims HBM in large blocks (cudaMalloc once per
// block, kept until the arena is destroyed) and hands out sub-ranges:
//   * best fit over the free ranges (a size-ordered multimap), the rest of
//     the range kept free;
//   * a freed range merges with its free neighbours inside the same block
//     (an address-ordered map), so mixed mesh sizes do not splinter the
//     blocks;
//   * ranges are multiples of 256 bytes, 256-byte aligned like cudaMalloc's,
//     which the tensor maps (16-byte base) and vector loads rely on;
//   * when no free range fits, a new block of max(request, growth step) is
//     claimed from the driver.
// The arena knows nothing of streams: a range must not be freed while queued
// work may still touch it. Contexts synchronise their own streams before
// they release buffers (ctx_release in engine.cu). All calls are thread-safe.
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "engine_internal.cuh"

namespace tpm {

struct DeviceArena {
  int device = 0;
  int64_t step = 1ll << 30;  // growth block size
  std::mutex mu;
  std::map<char *, size_t> blocks;            // base -> bytes
  std::map<char *, size_t> free_by_addr;      // free ranges
  std::multimap<size_t, char *> free_by_size;
  std::unordered_map<char *, size_t> used;    // allocated ranges
  int64_t reserved = 0, in_use = 0;
};

namespace {

constexpr size_t kAlign = 256;

char *block_of(DeviceArena *a, char *p) {
  auto it = a->blocks.upper_bound(p);
  return it == a->blocks.begin() ? nullptr : std::prev(it)->first;
}

void erase_free_by_size(DeviceArena *a, char *p, size_t n) {
  auto r = a->free_by_size.equal_range(n);
  for (auto it = r.first; it != r.second; ++it)
    if (it->second == p) {
      a->free_by_size.erase(it);
      return;
    }
}

void insert_free(DeviceArena *a, char *p, size_t n) {
  a->free_by_addr[p] = n;
  a->free_by_size.emplace(n, p);
}

// Claims a new block of at least n bytes from the driver (a->mu held).
cudaError_t grow(DeviceArena *a, size_t n) {
  size_t bytes = n > (size_t)a->step ? n : (size_t)a->step;
  bytes = (bytes + kAlign - 1) / kAlign * kAlign;
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e;
  }
  a->blocks[(char *)p] = bytes;
  a->reserved += (int64_t)bytes;
  insert_free(a, (char *)p, bytes);
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
  for (auto &b : a->blocks) cudaFree(b.first);
  cudaSetDevice(prev);
  delete a;
}

cudaError_t arena_reserve(DeviceArena *a, int64_t bytes) {
  std::lock_guard<std::mutex> lk(a->mu);
  if (bytes <= a->reserved - a->in_use) return cudaSuccess;
  return grow(a, (size_t)(bytes - (a->reserved - a->in_use)));
}

void arena_usage(DeviceArena *a, int64_t *reserved, int64_t *in_use) {
  std::lock_guard<std::mutex> lk(a->mu);
  if (reserved) *reserved = a->reserved;
  if (in_use) *in_use = a->in_use;
}

cudaError_t arena_alloc(DeviceArena *a, void **out, size_t bytes) {
  *out = nullptr;
  size_t n = (bytes + kAlign - 1) / kAlign * kAlign;
  if (n == 0) n = kAlign;
  std::lock_guard<std::mutex> lk(a->mu);
  auto it = a->free_by_size.lower_bound(n);
  if (it == a->free_by_size.end()) {
    cudaError_t e = grow(a, n);
    if (e != cudaSuccess) return e;
    it = a->free_by_size.lower_bound(n);
  }
  char *p = it->second;
  size_t have = it->first;
  a->free_by_size.erase(it);
  a->free_by_addr.erase(p);
  if (have > n) insert_free(a, p + n, have - n);
  a->used[p] = n;
  a->in_use += (int64_t)n;
  *out = p;
  return cudaSuccess;
}

void arena_free(DeviceArena *a, void *ptr) {
  if (!ptr) return;
  char *p = (char *)ptr;
  std::lock_guard<std::mutex> lk(a->mu);
  auto u = a->used.find(p);
  if (u == a->used.end()) return;
  size_t n = u->second;
  a->used.erase(u);
  a->in_use -= (int64_t)n;
  char *blk = block_of(a, p);
  // merge with the free range that ends at p and the one that starts at p + n
  auto next = a->free_by_addr.lower_bound(p);
  if (next != a->free_by_addr.begin()) {
    auto prev = std::prev(next);
    if (prev->first + prev->second == p && block_of(a, prev->first) == blk) {
      erase_free_by_size(a, prev->first, prev->second);
      p = prev->first;
      n += prev->second;
      a->free_by_addr.erase(prev);
    }
  }
  next = a->free_by_addr.find(p + n);
  if (next != a->free_by_addr.end() && block_of(a, next->first) == blk) {
    erase_free_by_size(a, next->first, next->second);
    n += next->second;
    a->free_by_addr.erase(next);
  }
  insert_free(a, p, n);
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
