// First-fit range allocator for the server's device pool: hands out [off,
// off + n) ranges of [0, size) and coalesces released ranges with their free
// neighbours.  Host-only, not thread-safe (the server calls it under its lock).
#pragma once

#include <stddef.h>

#include <iterator>
#include <map>

namespace tk {

class Pool {
 public:
  void init(size_t n) {
    free_.clear();
    free_[0] = n;
  }
  bool alloc(size_t n, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const size_t rest = it->second - n, o = it->first;
      free_.erase(it);
      if (rest) free_[o + n] = rest;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  // Free ranges in address order (tests and diagnostics).
  const std::map<size_t, size_t>& free_ranges() const { return free_; }

 private:
  std::map<size_t, size_t> free_;  // offset -> length, disjoint, never adjacent
};

}  // namespace tk
