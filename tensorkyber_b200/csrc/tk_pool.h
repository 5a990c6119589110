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
  // Next fit from `from` (the end of the previous allocation): [from, from +
  // n) when it is free, else the first free range after from that fits, else
  // the first fit from the start.  Requests that are admitted one after
  // another and finish roughly in order so get consecutive ranges.
  bool alloc_from(size_t n, size_t from, size_t* off) {
    auto it = free_.upper_bound(from);
    if (it != free_.begin()) {
      auto pv = std::prev(it);  // the free range starting at or before from
      const size_t o = pv->first, len = pv->second;
      if (from < o + len && o + len - from >= n) {
        if (from > o)
          pv->second = from - o;  // the part before from stays free
        else
          free_.erase(pv);
        if (o + len > from + n) free_[from + n] = o + len - from - n;
        *off = from;
        return true;
      }
    }
    for (; it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const size_t rest = it->second - n, o = it->first;
      free_.erase(it);
      if (rest) free_[o + n] = rest;
      return true;
    }
    return alloc(n, off);
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
