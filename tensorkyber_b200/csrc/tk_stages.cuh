// tk_stages.cuh -- the two matrix stages of the NTT on int8 mma.sync tiles,
// shared by the batched TMA kernels (tk_ntt_mma.cu) and the fused
// matrix-vector kernel (tk_matvec.cu).  Operand layouts and limb/byte
// conventions are those of tk_tables.h.
#pragma once
#include <stdint.h>

#include "tk_ptx.cuh"

namespace tk {

constexpr int kRowBytes = 528;  // one polynomial in shared memory: 512 B + 16 B pad

// ------------------------------------------------ shared building blocks ----
// Stage over m (forward stage 1 / inverse stage B) of one polynomial whose B
// operands (ldmatrix.trans of the natural-order row) are b0..b3.
template <bool kInverse>
__device__ __forceinline__ void stage_m(const uint32_t (&a)[2][4], int32_t c_lo, int32_t c_hi,
                                        uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3,
                                        uint8_t* row, uint32_t w_even, uint32_t w_odd,
                                        uint32_t w_nat, const uint32_t (&add)[4]) {
  const int32_t cinit[4] = {c_lo, c_lo, c_hi, c_hi};
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k32(lo0, a[0], b0, b1, cinit);
  mma_k32(hi0, a[1], b0, b1, zero);
  mma_k32(lo1, a[0], b2, b3, cinit);
  mma_k32(hi1, a[1], b2, b3, zero);
  uint32_t y0[4], y1[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const uint32_t s0 = (uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7);
    const uint32_t s1 = (uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7);
    if (kInverse) {  // centred: accumulators carry +(q-1)/2
      y0[e] = red_exact(s0) - 1664u;
      y1[e] = red_exact(s1) - 1664u;
    } else {
      y0[e] = red_lazy(s0);
      y1[e] = red_lazy(s1);
    }
  }
  // D regs: [0] (row i, c=2q), [1] (row i, c=2q+1), [2]/[3] row i+8; n-tile 1 is c+8.
  if (kInverse) {  // natural order; plus the addend pairs (int16 wrap-around add)
    y0[0] += (uint32_t)(int32_t)(int16_t)(add[0] & 0xffffu);
    y0[1] += (uint32_t)((int32_t)add[0] >> 16);
    y1[0] += (uint32_t)(int32_t)(int16_t)(add[1] & 0xffffu);
    y1[1] += (uint32_t)((int32_t)add[1] >> 16);
    y0[2] += (uint32_t)(int32_t)(int16_t)(add[2] & 0xffffu);
    y0[3] += (uint32_t)((int32_t)add[2] >> 16);
    y1[2] += (uint32_t)(int32_t)(int16_t)(add[3] & 0xffffu);
    y1[3] += (uint32_t)((int32_t)add[3] >> 16);
    *(uint32_t*)(row + w_nat) = pack2(y0[0], y0[1]);
    *(uint32_t*)(row + w_nat + 16) = pack2(y1[0], y1[1]);
    *(uint32_t*)(row + w_nat + 256) = pack2(y0[2], y0[3]);
    *(uint32_t*)(row + w_nat + 256 + 16) = pack2(y1[2], y1[3]);
  } else {  // parity-split slots (c=2q | c=8+2q), (c=2q+1 | c=9+2q)
    *(uint32_t*)(row + w_even) = pack2(y0[0], y1[0]);
    *(uint32_t*)(row + w_odd) = pack2(y0[1], y1[1]);
    *(uint32_t*)(row + w_even + 256) = pack2(y0[2], y1[2]);
    *(uint32_t*)(row + w_odd + 256) = pack2(y0[3], y1[3]);
  }
}

// Block-wise stage (forward stage 2 / inverse stage A) for blocks I, I+1 of 8
// polynomials.  r[0..3]: B operands (even I, odd I, even I+1, odd I+1).
// Output: natural order, polynomials 2q and 2q+1 of the n-tile.
template <bool kInverse>
__device__ __forceinline__ void stage_c(const uint32_t (&a)[2][2][2], const int32_t (&ca)[2][2],
                                        const uint32_t (&r)[4], uint8_t* out) {
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int32_t ce[4] = {ca[h][0], ca[h][0], 0, 0};
    const int32_t co[4] = {ca[h][1], ca[h][1], 0, 0};
    int32_t de[4], dodd[4];
    mma_k16(de, a[h][0], r[2 * h], ce);
    mma_k16(dodd, a[h][1], r[2 * h + 1], co);
    const uint32_t se0 = (uint32_t)de[0] + ((uint32_t)de[2] << 7);
    const uint32_t se1 = (uint32_t)de[1] + ((uint32_t)de[3] << 7);
    const uint32_t so0 = (uint32_t)dodd[0] + ((uint32_t)dodd[2] << 7);
    const uint32_t so1 = (uint32_t)dodd[1] + ((uint32_t)dodd[3] << 7);
    uint32_t e0, e1, o0, o1;
    if (kInverse) {
      e0 = red_lazy(se0); e1 = red_lazy(se1); o0 = red_lazy(so0); o1 = red_lazy(so1);
    } else {
      e0 = red_exact(se0); e1 = red_exact(se1); o0 = red_exact(so0); o1 = red_exact(so1);
    }
    *(uint32_t*)(out + 32 * h) = pack2(e0, o0);
    *(uint32_t*)(out + kRowBytes + 32 * h) = pack2(e1, o1);
  }
}

}  // namespace tk
