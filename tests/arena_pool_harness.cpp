// C entry points over tpm::RangePool (lageunha_b200/csrc/arena_core.h) for
// tests/test_arena_pool.py, which compiles this file with the host compiler.
// Addresses are plain numbers here: the pool never touches the memory.
#include "arena_core.h"

using tpm::RangePool;

extern "C" {
void *pool_new() { return new RangePool(); }
void pool_delete(void *p) { delete static_cast<RangePool *>(p); }
void pool_add_block(void *p, uint64_t base, uint64_t bytes) {
  static_cast<RangePool *>(p)->add_block(reinterpret_cast<char *>(base), (size_t)bytes);
}
uint64_t pool_alloc(void *p, uint64_t bytes) {
  return reinterpret_cast<uint64_t>(static_cast<RangePool *>(p)->alloc((size_t)bytes));
}
int pool_release(void *p, uint64_t addr) {
  return static_cast<RangePool *>(p)->release(reinterpret_cast<char *>(addr)) ? 1 : 0;
}
// [0] reserved bytes [1] bytes in use [2] free ranges [3] largest free range
void pool_stats(void *p, int64_t *out) {
  const RangePool *r = static_cast<RangePool *>(p);
  out[0] = r->reserved();
  out[1] = r->in_use();
  out[2] = (int64_t)r->free_ranges();
  out[3] = (int64_t)r->largest_free();
}
}
