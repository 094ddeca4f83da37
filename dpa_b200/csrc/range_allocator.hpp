// range_allocator.hpp -- first-fit allocator of [0, capacity) ranges for the
// request server's arenas (particle slots, curve-staging vertices). Host code
// only; the CPU tests compile it on its own.
#pragma once

#include <cstdint>
#include <iterator>
#include <map>

namespace dpa {

// Free ranges are kept maximal (adjacent ones merge on release), so the first
// free range long enough is the lowest-addressed place a request fits.
class range_allocator {
 public:
  explicit range_allocator(uint64_t capacity = 0) { reset(capacity); }
  void reset(uint64_t capacity) {
    free_.clear();
    if (capacity) free_[0] = capacity;
  }
  // The lowest offset with n free entries after it; false when none has.
  bool allocate(uint64_t n, uint64_t* offset) {
    if (n == 0) {
      *offset = 0;
      return true;
    }
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *offset = it->first;
        const uint64_t rest = it->second - n;
        const uint64_t at = it->first + n;
        free_.erase(it);
        if (rest) free_[at] = rest;
        return true;
      }
    }
    return false;
  }
  // Returns [offset, offset + n), which allocate handed out.
  void release(uint64_t offset, uint64_t n) {
    if (n == 0) return;
    auto next = free_.lower_bound(offset);
    if (next != free_.end() && offset + n == next->first) {
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == offset) {
        prev->second += n;
        return;
      }
    }
    free_[offset] = n;
  }
  // Free ranges, lowest first: offset -> length.
  const std::map<uint64_t, uint64_t>& free_ranges() const { return free_; }

 private:
  std::map<uint64_t, uint64_t> free_;
};

}  // namespace dpa
