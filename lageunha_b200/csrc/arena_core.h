// The device arena's range bookkeeping, free of CUDA so that it can be
// tested on the host: blocks of address space are added, ranges are handed
// out best fit (the smallest free range that holds the request, the rest of
// it kept free), and a released range merges with its free neighbours in the
// same block. Ranges are multiples of kRangeAlign bytes and start at
// multiples of it when the blocks do. Not thread-safe: the caller locks.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <iterator>
#include <map>
#include <unordered_map>

namespace tpm {

constexpr size_t kRangeAlign = 256;

class RangePool {
 public:
  // Adds [base, base + bytes) as a free block (bytes a multiple of kRangeAlign).
  void add_block(char *base, size_t bytes) {
    blocks_[base] = bytes;
    reserved_ += (int64_t)bytes;
    insert_free(base, bytes);
  }

  // The request rounded up to whole ranges (at least one).
  static size_t round(size_t bytes) {
    size_t n = (bytes + kRangeAlign - 1) / kRangeAlign * kRangeAlign;
    return n ? n : kRangeAlign;
  }

  // A range of round(bytes), or nullptr when no free range holds it.
  char *alloc(size_t bytes) {
    size_t n = round(bytes);
    auto it = free_by_size_.lower_bound(n);
    if (it == free_by_size_.end()) return nullptr;
    char *p = it->second;
    size_t have = it->first;
    free_by_size_.erase(it);
    free_by_addr_.erase(p);
    if (have > n) insert_free(p + n, have - n);
    used_[p] = n;
    in_use_ += (int64_t)n;
    return p;
  }

  // Releases a range alloc returned; anything else is ignored (returns false).
  bool release(char *p) {
    auto u = used_.find(p);
    if (u == used_.end()) return false;
    size_t n = u->second;
    used_.erase(u);
    in_use_ -= (int64_t)n;
    char *blk = block_of(p);
    // merge with the free range that ends at p and the one that starts at p + n
    auto next = free_by_addr_.lower_bound(p);
    if (next != free_by_addr_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == p && block_of(prev->first) == blk) {
        erase_free_by_size(prev->first, prev->second);
        p = prev->first;
        n += prev->second;
        free_by_addr_.erase(prev);
      }
    }
    next = free_by_addr_.find(p + n);
    if (next != free_by_addr_.end() && block_of(next->first) == blk) {
      erase_free_by_size(next->first, next->second);
      n += next->second;
      free_by_addr_.erase(next);
    }
    insert_free(p, n);
    return true;
  }

  int64_t reserved() const { return reserved_; }
  int64_t in_use() const { return in_use_; }
  size_t free_ranges() const { return free_by_addr_.size(); }
  size_t largest_free() const { return free_by_size_.empty() ? 0 : free_by_size_.rbegin()->first; }
  const std::map<char *, size_t> &blocks() const { return blocks_; }

 private:
  char *block_of(char *p) const {
    auto it = blocks_.upper_bound(p);
    return it == blocks_.begin() ? nullptr : std::prev(it)->first;
  }
  void erase_free_by_size(char *p, size_t n) {
    auto r = free_by_size_.equal_range(n);
    for (auto it = r.first; it != r.second; ++it)
      if (it->second == p) {
        free_by_size_.erase(it);
        return;
      }
  }
  void insert_free(char *p, size_t n) {
    free_by_addr_[p] = n;
    free_by_size_.emplace(n, p);
  }

  std::map<char *, size_t> blocks_;        // base -> bytes
  std::map<char *, size_t> free_by_addr_;  // free ranges
  std::multimap<size_t, char *> free_by_size_;
  std::unordered_map<char *, size_t> used_;  // allocated ranges
  int64_t reserved_ = 0, in_use_ = 0;
};

}  // namespace tpm
