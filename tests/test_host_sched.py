"""The host-buffer transforms' chunk schedule (tk_host_sched.h), on the CPU:
chunks cover the batch exactly, never exceed the cap, start short and end
short (the copies nothing overlaps), and leave no sliver below the ramp size
behind whenever the cap allows it."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <stdio.h>
#include <vector>
#include "tk_host_sched.h"

using tk::host_chunk_size;
using tk::kHostRampPolys;

static int fail(const char* what, size_t npoly, size_t chunk) {
  printf("FAIL %s npoly=%zu chunk=%zu\n", what, npoly, chunk);
  return 1;
}

int main() {
  const size_t caps[] = {1, 1000, 4096, 8192, 32768};
  std::vector<size_t> sizes;
  for (size_t n = 1; n <= 70000; n++) sizes.push_back(n);
  for (size_t n = 70000; n <= ((size_t)3 << 20); n += 4099) sizes.push_back(n);
  sizes.push_back((size_t)1 << 18);
  sizes.push_back((size_t)1 << 20);
  for (size_t cap : caps)
    for (size_t npoly : sizes) {
      if (cap < kHostRampPolys && npoly > 20000) continue;  // tiny caps: small batches only
      std::vector<size_t> ch;
      size_t done = 0;
      for (int c = 0; done < npoly; c++) {
        const size_t rem = npoly - done, n = host_chunk_size(c, rem, cap);
        if (n < 1 || n > rem || n > cap) return fail("chunk bounds", npoly, cap);
        ch.push_back(n);
        done += n;
        if (ch.size() > npoly + 64) return fail("no progress", npoly, cap);
      }
      if (done != npoly) return fail("coverage", npoly, cap);
      if (cap >= 2 * kHostRampPolys) {
        // no sliver: every chunk but a lone one is at least the ramp size
        for (size_t n : ch)
          if (ch.size() > 1 && n < kHostRampPolys) return fail("sliver", npoly, cap);
        // short head and tail around full-size chunks
        if (npoly >= 4 * kHostRampPolys) {
          if (ch.front() != kHostRampPolys) return fail("head", npoly, cap);
          if (ch.back() >= 2 * kHostRampPolys) return fail("tail", npoly, cap);
        }
        // the middle reaches the cap on long batches
        if (npoly >= 8 * cap) {
          size_t mx = 0;
          for (size_t n : ch) mx = n > mx ? n : mx;
          if (mx != cap) return fail("full chunks", npoly, cap);
        }
      }
    }
  // the headline batch with the default 16 MiB cap: a short list of chunks
  size_t done = 0, count = 0;
  for (int c = 0; done < ((size_t)1 << 18); c++, count++)
    done += host_chunk_size(c, ((size_t)1 << 18) - done, 32768);
  if (count > 16) return fail("chunk count", (size_t)1 << 18, 32768);
  printf("ok %zu\n", count);
  return 0;
}
"""


def test_host_chunk_schedule_properties(tmp_path):
    src = tmp_path / "sched_driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "sched_driver"
    p = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror",
                        "-I", os.path.join(ROOT, "tensorkyber_b200", "csrc"), str(src),
                        "-o", str(exe)], capture_output=True, text=True, timeout=180)
    assert p.returncode == 0, p.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
