"""The server's device-pool allocator (tk_pool.h), driven on the CPU against
a reference model: every range it hands out is the first free range that
fits, lies inside the pool and overlaps nothing live; its free list stays
sorted, disjoint and coalesced, and equals the complement of the live ranges;
releasing everything restores one free range."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <stdio.h>
#include <stdlib.h>
#include <iterator>
#include <map>
#include <random>
#include <vector>
#include "tk_pool.h"

static int fail(const char* what, long step) { printf("FAIL %s at %ld\n", what, step); return 1; }

int main() {
  const size_t kSize = 1 << 20;
  std::mt19937_64 rng(20241204);
  for (int round = 0; round < 4; round++) {
    tk::Pool P;
    P.init(kSize);
    std::map<size_t, size_t> live;  // offset -> length
    for (long step = 0; step < 50000; step++) {
      const bool do_alloc = live.empty() || (rng() % 100) < (round == 3 ? 45u : 55u);
      if (do_alloc) {
        const size_t n = 1 + rng() % (round == 0 ? 64 : kSize / 16);
        // expected: first gap (by offset) of length >= n in the complement of live
        size_t want = (size_t)-1, cur = 0;
        for (auto& r : live) {
          if (r.first - cur >= n) { want = cur; break; }
          cur = r.first + r.second;
        }
        if (want == (size_t)-1 && kSize - cur >= n) want = cur;
        size_t off = 0;
        const bool ok = P.alloc(n, &off);
        if (ok != (want != (size_t)-1)) return fail("alloc success", step);
        if (ok) {
          if (off != want) return fail("first fit", step);
          if (off + n > kSize) return fail("bounds", step);
          live[off] = n;
        }
      } else {
        auto it = live.begin();
        std::advance(it, rng() % live.size());
        P.release(it->first, it->second);
        live.erase(it);
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
