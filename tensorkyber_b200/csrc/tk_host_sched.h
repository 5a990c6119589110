// Chunk schedule of the host-buffer transforms (tk_ntt_host / tk_invntt_host).
// Chunks of at most `chunk` polynomials: the first ones grow from
// kHostRampPolys (doubling) and the last ones shrink towards it (at most half
// of what remains), because the first upload and the last download run with
// nothing beside them; a remainder below kHostRampPolys is never left behind
// when the rest fits one chunk.  Host-only.
#pragma once

#include <stddef.h>

namespace tk {

constexpr size_t kHostRampPolys = 4096;

// Size of chunk c (0-based) when `remaining` polynomials are left.
inline size_t host_chunk_size(int c, size_t remaining, size_t chunk) {
  size_t n = chunk;
  if (c < 16 && (kHostRampPolys << c) < n) n = kHostRampPolys << c;
  const size_t half = (remaining + 1) / 2;
  const size_t tail = half > kHostRampPolys ? half : kHostRampPolys;
  if (tail < n) n = tail;
  if (remaining - n < kHostRampPolys && remaining <= chunk) n = remaining;  // no sliver
  return n < remaining ? n : remaining;
}

}  // namespace tk
