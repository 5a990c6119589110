"""The server's device-pool allocator (tk_pool.h), driven on the CPU against
a reference model: every range it hands out is the one its policy names
(first fit for alloc; for alloc_from, the hint itself when it starts room
enough, else the first free range after it that fits, else the first fit),
lies inside the pool and overlaps nothing live; its free list stays sorted,
disjoint and coalesced, and equals the complement of the live ranges;
releasing everything restores one free range.  With releases in allocation
order (the server's requests finish roughly so), next fit hands out
consecutive ranges."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <stdio.h>
#include <stdlib.h>
#include <algorithm>
#include <iterator>
#include <map>
#include <random>
#include <vector>
#include "tk_pool.h"

static int fail(const char* what, long step) { printf("FAIL %s at %ld\n", what, step); return 1; }

int main() {
  const size_t kSize = 1 << 20;
  std::mt19937_64 rng(20241204);
  long adjacent = 0, fifo_allocs = 0;
  for (int round = 0; round < 8; round++) {
    const bool next_fit = round >= 4, fifo = round >= 6;
    tk::Pool P;
    P.init(kSize);
    std::map<size_t, size_t> live;  // offset -> length
    std::vector<size_t> order;      // live offsets in allocation order (fifo rounds)
    size_t hint = 0;                // end of the last allocation
    for (long step = 0; step < 50000; step++) {
      const bool do_alloc = live.empty() || (rng() % 100) < (round % 4 == 3 ? 45u : 55u);
      if (do_alloc) {
        const size_t n = 1 + rng() % (round % 4 == 0 ? 64 : kSize / 16);
        // the gaps (complement of live), by offset
        std::vector<std::pair<size_t, size_t>> gaps;
        size_t cur = 0;
        for (auto& r : live) {
          if (r.first > cur) gaps.push_back({cur, r.first});
          cur = r.first + r.second;
        }
        if (cur < kSize) gaps.push_back({cur, kSize});
        size_t want = (size_t)-1;
        if (next_fit) {
          for (auto& g : gaps)  // the hint inside a gap with room
            if (g.first <= hint && hint < g.second && g.second - hint >= n) want = hint;
          if (want == (size_t)-1)
            for (auto& g : gaps)
              if (g.first > hint && g.second - g.first >= n) { want = g.first; break; }
        }
        if (want == (size_t)-1)
          for (auto& g : gaps)
            if (g.second - g.first >= n) { want = g.first; break; }
        size_t off = 0;
        const bool ok = next_fit ? P.alloc_from(n, hint, &off) : P.alloc(n, &off);
        if (ok != (want != (size_t)-1)) return fail("alloc success", step);
        if (ok) {
          if (off != want) return fail(next_fit ? "next fit" : "first fit", step);
          if (off + n > kSize) return fail("bounds", step);
          if (fifo) {
            fifo_allocs++;
            adjacent += off == hint;
          }
          live[off] = n;
          order.push_back(off);
          hint = off + n;
        }
      } else {
        // fifo rounds: mostly the oldest live range, as requests finish
        size_t victim;
        if (fifo && rng() % 8 != 0) {
          victim = order.front();
        } else {
          auto it = live.begin();
          std::advance(it, rng() % live.size());
          victim = it->first;
        }
        order.erase(std::find(order.begin(), order.end(), victim));
        P.release(victim, live[victim]);
        live.erase(victim);
      }
      // the free list is the complement of live: sorted, disjoint, coalesced
      size_t cur = 0;
      auto f = P.free_ranges().begin();
      for (auto& r : live) {
        if (r.first > cur) {
          if (f == P.free_ranges().end() || f->first != cur || f->second != r.first - cur)
            return fail("free list", step);
          ++f;
        }
        if (r.first < cur) return fail("overlap", step);
        cur = r.first + r.second;
      }
      if (cur < kSize) {
        if (f == P.free_ranges().end() || f->first != cur || f->second != kSize - cur)
          return fail("free tail", step);
        ++f;
      }
      if (f != P.free_ranges().end()) return fail("extra free range", step);
    }
    while (!live.empty()) {
      P.release(live.begin()->first, live.begin()->second);
      live.erase(live.begin());
    }
    if (P.free_ranges().size() != 1 || P.free_ranges().begin()->first != 0 ||
        P.free_ranges().begin()->second != kSize)
      return fail("full recovery", -1);
  }
  // with releases in allocation order, next fit keeps most neighbours adjacent
  if (adjacent * 10 < fifo_allocs * 6) {
    printf("FAIL adjacency %ld of %ld\n", adjacent, fifo_allocs);
    return 1;
  }
  printf("ok\n");
  return 0;
}
"""


def test_pool_against_reference_model(tmp_path):
    src = tmp_path / "pool_driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "pool_driver"
    p = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror",
                        "-I", os.path.join(ROOT, "tensorkyber_b200", "csrc"), str(src),
                        "-o", str(exe)], capture_output=True, text=True, timeout=180)
    assert p.returncode == 0, p.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
