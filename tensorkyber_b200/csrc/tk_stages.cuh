// tk_stages.cuh -- the two matrix stages of the NTT on int8 mma.sync tiles,
// shared by the batched TMA kernels (tk_ntt_mma.cu) and the fused
// matrix-vector kernel (tk_matvec.cu).  Operand layouts and limb/byte
// conventions are those of tk_tables.h.
#pragma once
#include <stdint.h>

#include "tk_ptx.cuh"

namespace tk {

constexpr int kRowBytes = 528;  // one polynomial in shared memory: 512 B + 16 B pad
// one polynomial of int32 stage-1 sums (the "wide" kernels): 1024 B + 16 B pad
constexpr int kWideRowBytes = 1040;

// ------------------------------------------------ shared building blocks ----
template <bool kInverse, bool kAdd>
__device__ __forceinline__ void stage_m_out(const int32_t (&lo0)[4], const int32_t (&hi0)[4],
                                            const int32_t (&lo1)[4], const int32_t (&hi1)[4],
                                            uint8_t* row, uint32_t w_even, uint32_t w_odd,
                                            uint32_t w_nat, const uint32_t (&add)[4]);

// Stage over m (forward stage 1 / inverse stage B) of one polynomial whose B
// operands (ldmatrix.trans of the natural-order row) are b0..b3.  Inverse
// with kAdd: the addend pairs `add` are added to the output (int16
// wrap-around); without it `add` is ignored.
// c0 / c1: the group-0 accumulator init of n-tiles 0 and 1 (D register order).
template <bool kInverse, bool kAdd = false>
__device__ __forceinline__ void stage_m_q(const uint32_t (&a)[2][4], const int32_t (&c0)[4],
                                          const int32_t (&c1)[4], uint32_t b0, uint32_t b1,
                                          uint32_t b2, uint32_t b3, uint8_t* row, uint32_t w_even,
                                          uint32_t w_odd, uint32_t w_nat,
                                          const uint32_t (&add)[4]) {
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k32(lo0, a[0], b0, b1, c0);
  mma_k32(hi0, a[1], b0, b1, zero);
  mma_k32(lo1, a[0], b2, b3, c1);
  mma_k32(hi1, a[1], b2, b3, zero);
  stage_m_out<kInverse, kAdd>(lo0, hi0, lo1, hi1, row, w_even, w_odd, w_nat, add);
}
// The same with one init per row half (rows lane/4 and lane/4 + 8).
template <bool kInverse, bool kAdd = false>
__device__ __forceinline__ void stage_m(const uint32_t (&a)[2][4], int32_t c_lo, int32_t c_hi,
                                        uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3,
                                        uint8_t* row, uint32_t w_even, uint32_t w_odd,
                                        uint32_t w_nat, const uint32_t (&add)[4]) {
  const int32_t cinit[4] = {c_lo, c_lo, c_hi, c_hi};
  stage_m_q<kInverse, kAdd>(a, cinit, cinit, b0, b1, b2, b3, row, w_even, w_odd, w_nat, add);
}

// Epilogue of the stage over m from its accumulators (lo / hi limb, n-tiles 0
// and 1): forward lazy reduction to parity-split rows; inverse exact reduction,
// centring and (kAdd) the addend, natural order.
template <bool kInverse, bool kAdd>
__device__ __forceinline__ void stage_m_out(const int32_t (&lo0)[4], const int32_t (&hi0)[4],
                                            const int32_t (&lo1)[4], const int32_t (&hi1)[4],
                                            uint8_t* row, uint32_t w_even, uint32_t w_odd,
                                            uint32_t w_nat, const uint32_t (&add)[4]) {
  uint32_t y0[4], y1[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const uint32_t s0 = (uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7);
    const uint32_t s1 = (uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7);
    if (kInverse) {  // centred
      y0[e] = red_centred(s0);
      y1[e] = red_centred(s1);
    } else {
      y0[e] = red_lazy(s0);
      y1[e] = red_lazy(s1);
    }
  }
  // D regs: [0] (row i, c=2q), [1] (row i, c=2q+1), [2]/[3] row i+8; n-tile 1 is c+8.
  if (kInverse) {  // natural order; plus the addend pairs (int16 wrap-around add)
    if (kAdd) {
    y0[0] += (uint32_t)(int32_t)(int16_t)(add[0] & 0xffffu);
    y0[1] += (uint32_t)((int32_t)add[0] >> 16);
    y1[0] += (uint32_t)(int32_t)(int16_t)(add[1] & 0xffffu);
    y1[1] += (uint32_t)((int32_t)add[1] >> 16);
    y0[2] += (uint32_t)(int32_t)(int16_t)(add[2] & 0xffffu);
    y0[3] += (uint32_t)((int32_t)add[2] >> 16);
    y1[2] += (uint32_t)(int32_t)(int16_t)(add[3] & 0xffffu);
    y1[3] += (uint32_t)((int32_t)add[3] >> 16);
    }
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

// Forward stage 1 without the reduction (the "wide" kernels): S = D_lo +
// 128 D_hi, non-negative and below 2^25, goes to the polynomial's int32
// intermediate row `irow` as it is; forward stage 2 then reads its four bytes
// (stage_c_wide).  Row layout: block i at 64 i, its parity-s half (8 values,
// slot order of FwdFrags::s2) at 32 (s ^ ((i >> 1) & 1)) -- the xor spreads
// one store instruction's 8-byte lanes over all banks.  w_e / w_o: this
// lane's offsets of block lane/4, even / odd half, slots 2q and 2q+1.
__device__ __forceinline__ void stage_m_wide(const uint32_t (&a)[2][4], int32_t c_lo,
                                             int32_t c_hi, uint32_t b0, uint32_t b1, uint32_t b2,
                                             uint32_t b3, uint8_t* irow, uint32_t w_e,
                                             uint32_t w_o) {
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
    y0[e] = (uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7);
    y1[e] = (uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7);
  }
  // D regs: [0] (block i, c=2q), [1] (i, c=2q+1), [2]/[3] block i+8; n-tile 1 is c+8
  *(uint2*)(irow + w_e) = make_uint2(y0[0], y1[0]);
  *(uint2*)(irow + w_o) = make_uint2(y0[1], y1[1]);
  *(uint2*)(irow + w_e + 512) = make_uint2(y0[2], y1[2]);
  *(uint2*)(irow + w_o + 512) = make_uint2(y0[3], y1[3]);
}

// Inverse stage B from int32 intermediates (the "wide" kernels): b[t] = the
// two m16n8k32 B operand pairs of n-tile t (c = 8t .. 8t+7) for blocks m =
// 0-7 and 8-15, each 32-bit word one stage-A sum S; the two K chunks
// accumulate into one accumulator per limb.  Output as stage_m<true, kAdd>.
template <bool kAdd>
__device__ __forceinline__ void stage_m_inv_wide(const uint32_t (&a)[2][2][4],
                                                 const int32_t (&c)[2][4],
                                                 const uint32_t (&b)[2][4], uint8_t* row,
                                                 uint32_t w_nat, const uint32_t (&add)[4]) {
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k32(lo0, a[0][0], b[0][0], b[0][1], c[0]);
  mma_k32(hi0, a[1][0], b[0][0], b[0][1], zero);
  mma_k32(lo1, a[0][0], b[1][0], b[1][1], c[1]);
  mma_k32(hi1, a[1][0], b[1][0], b[1][1], zero);
  mma_k32(lo0, a[0][1], b[0][2], b[0][3], lo0);
  mma_k32(hi0, a[1][1], b[0][2], b[0][3], hi0);
  mma_k32(lo1, a[0][1], b[1][2], b[1][3], lo1);
  mma_k32(hi1, a[1][1], b[1][2], b[1][3], hi1);
  stage_m_out<true, kAdd>(lo0, hi0, lo1, hi1, row, 0, 0, w_nat, add);
}

// Forward stage 1 in single-limb form, for inputs in [-128, 127]: one data
// byte per coefficient (x + 128) instead of two, so half the MMA work of
// stage_m.  bt0 / bt1: the m16n8k16 B operands of n-tiles 0 and 1 (c = lane/4
// and 8 + lane/4), byte j of lane t = lane%4 holding block
// m = {2t, 2t+1, 8+2t, 9+2t}[j] -- the order of the low bytes in stage_m's
// k32 fragments, which FwdFrags::s1b's column order follows.  Output as
// stage_m<false>: lazy Barrett, parity-split rows.
__device__ __forceinline__ void stage_m_small(const uint32_t (&a)[2][2], int32_t c_lo,
                                              int32_t c_hi, uint32_t bt0, uint32_t bt1,
                                              uint8_t* row, uint32_t w_even, uint32_t w_odd) {
  const int32_t cinit[4] = {c_lo, c_lo, c_hi, c_hi};
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k16(lo0, a[0], bt0, cinit);
  mma_k16(hi0, a[1], bt0, zero);
  mma_k16(lo1, a[0], bt1, cinit);
  mma_k16(hi1, a[1], bt1, zero);
  uint32_t y0[4], y1[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    y0[e] = red_lazy((uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7));
    y1[e] = red_lazy((uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7));
  }
  *(uint32_t*)(row + w_even) = pack2(y0[0], y1[0]);
  *(uint32_t*)(row + w_odd) = pack2(y0[1], y1[1]);
  *(uint32_t*)(row + w_even + 256) = pack2(y0[2], y1[2]);
  *(uint32_t*)(row + w_odd + 256) = pack2(y0[3], y1[3]);
}

// stage_m_small without the reduction (the "wide" kernels): the sums S (below
// 2^24: one data byte x + 128 per coefficient) go to the int32 intermediate
// row as stage_m_wide stores them.
__device__ __forceinline__ void stage_m_small_wide(const uint32_t (&a)[2][2], int32_t c_lo,
                                                   int32_t c_hi, uint32_t bt0, uint32_t bt1,
                                                   uint8_t* irow, uint32_t w_e, uint32_t w_o) {
  const int32_t cinit[4] = {c_lo, c_lo, c_hi, c_hi};
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k16(lo0, a[0], bt0, cinit);
  mma_k16(hi0, a[1], bt0, zero);
  mma_k16(lo1, a[0], bt1, cinit);
  mma_k16(hi1, a[1], bt1, zero);
  uint32_t y0[4], y1[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    y0[e] = (uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7);
    y1[e] = (uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7);
  }
  *(uint2*)(irow + w_e) = make_uint2(y0[0], y1[0]);
  *(uint2*)(irow + w_o) = make_uint2(y0[1], y1[1]);
  *(uint2*)(irow + w_e + 512) = make_uint2(y0[2], y1[2]);
  *(uint2*)(irow + w_o + 512) = make_uint2(y0[3], y1[3]);
}

// The single-limb B operands from stage_m's two k32 fragment registers of one
// n-tile (int16 inputs): low bytes, biased to x + 128.  *bad collects bits
// where a high byte is not the sign extension of its low byte (input outside
// [-128, 127]).
__device__ __forceinline__ uint32_t small_operand(uint32_t b0, uint32_t b1, uint32_t* bad) {
  const uint32_t lo = __byte_perm(b0, b1, 0x6420);
  const uint32_t hi = __byte_perm(b0, b1, 0x7531);
  *bad |= hi ^ (((lo >> 7) & 0x01010101u) * 0xffu);
  return lo ^ 0x80808080u;
}

// The single-limb B operand of one n-tile from packed fields: w0..w3 hold
// the packed bytes of blocks m = 2t, 2t+1, 8+2t, 9+2t; byte `sel` (a
// __byte_perm selector picking byte k of the first and second word) of each
// holds the field at bit `shift`.  Fields are kBits-bit two's complement; the
// result byte is value + 128 = (field ^ sign bit) + 128 - 2^(kBits-1).
template <int kBits>
__device__ __forceinline__ uint32_t packed_operand(uint32_t w0, uint32_t w1, uint32_t w2,
                                                   uint32_t w3, uint32_t sel, uint32_t shift) {
  constexpr uint32_t kMask = ((1u << kBits) - 1u) * 0x01010101u;
  constexpr uint32_t kSign = (1u << (kBits - 1)) * 0x01010101u;
  constexpr uint32_t kOff = (128u - (1u << (kBits - 1))) * 0x01010101u;
  const uint32_t g = __byte_perm(__byte_perm(w0, w1, sel), __byte_perm(w2, w3, sel), 0x5410);
  return (((g >> shift) & kMask) ^ kSign) + kOff;
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

// Forward stage 2 from int32 intermediates for blocks I, I+1 of 8
// polynomials: r[4h .. 4h+3] = B operands of block I+h (even k0-15, even
// k16-31, odd k0-15, odd k16-31), each 32-bit word one intermediate S.
// Output as stage_c<false>: exact reduction, natural order, polynomials 2q
// and 2q+1 of the n-tile.
__device__ __forceinline__ void stage_c_wide(const uint32_t (&a)[2][2][4], const uint32_t (&r)[8],
                                             uint8_t* out) {
  const int32_t zero[4] = {0, 0, 0, 0};
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int32_t de[4], dodd[4];
    mma_k32(de, a[h][0], r[4 * h], r[4 * h + 1], zero);
    mma_k32(dodd, a[h][1], r[4 * h + 2], r[4 * h + 3], zero);
    const uint32_t e0 = red_exact((uint32_t)de[0] + ((uint32_t)de[2] << 7));
    const uint32_t e1 = red_exact((uint32_t)de[1] + ((uint32_t)de[3] << 7));
    const uint32_t o0 = red_exact((uint32_t)dodd[0] + ((uint32_t)dodd[2] << 7));
    const uint32_t o1 = red_exact((uint32_t)dodd[1] + ((uint32_t)dodd[3] << 7));
    *(uint32_t*)(out + 32 * h) = pack2(e0, o0);
    *(uint32_t*)(out + kRowBytes + 32 * h) = pack2(e1, o1);
  }
}

// Inverse stage A of blocks I, I+1 for 8 polynomials into int32
// intermediates (the "wide" kernels).  x: biased, parity-split B operands as
// stage_c<true>.  The sums S (< 2^24) of output c' = 2(lane/4) + s of blocks I
// and I+1 go side by side (8 bytes) to polynomial 2q's row `rows` and 2q+1's
// row rows + kWideRowBytes at offset off[s].  Row layout: [c][m], c at 64 c,
// blocks m .. m+3 in the 16-byte chunk (m >> 2) ^ ((c >> 1) & 3) -- the xor
// keeps stage B's ldmatrix rows on distinct banks.
__device__ __forceinline__ void stage_c_inv_wide(const uint32_t (&a)[2][2][2],
                                                 const int32_t (&ca)[2][2], const uint32_t (&x)[4],
                                                 uint8_t* rows, const uint32_t (&off)[2]) {
  uint32_t S[2][2][2];  // [parity][polynomial 2q + j][block I + h]
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int32_t c[4] = {ca[h][s], ca[h][s], 0, 0};
      int32_t d[4];
      mma_k16(d, a[h][s], x[2 * h + s], c);
      S[s][0][h] = (uint32_t)d[0] + ((uint32_t)d[2] << 7);
      S[s][1][h] = (uint32_t)d[1] + ((uint32_t)d[3] << 7);
    }
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int j = 0; j < 2; j++)
      *(uint2*)(rows + j * kWideRowBytes + off[s]) = make_uint2(S[s][j][0], S[s][j][1]);
}

// ------------------------------------------------------------- basemul ----
constexpr uint32_t kRinv = 169;                 // 2^-16 mod q
constexpr uint32_t kSumBias = 3329u * 262144u;  // > 2^29.7 >= |sum|; sum + bias < 2^31

// Any S < 2^32: representative in [0, 1.41 q) ([0, 1.21 q) for S < 2^31).
// floor(S * 1290167 / 2^32) undershoots S / q by less than 0.41, so the
// quotient is at most one below floor(S / q).
__device__ __forceinline__ uint32_t red_wide(uint32_t s) {
  return s - __umulhi(s, 1290167u) * 3329u;
}

// One output polynomial of a job's basemul-accumulate for one lane, which
// owns coefficient pairs 4l .. 4l+3 (16 bytes of every polynomial): a[j] =
// those bytes of A_ij (any int16), b[j] = of ntt(s_j) (in [0, q)), zr = the
// pairs' constants z_t * 2^-16.  The raw products are accumulated first, per
// pair t with z = z_t:
//   out0 = 2^-16 (sum_j a0 b0 + z sum_j a1 b1),  out1 = 2^-16 sum_j (a0 b1 + a1 b0)
// so the constants are applied once per output pair.  |sum| < 2K * 32768 * q
// < 2^30 for K <= 4.  Output pairs in [0, 3q).
template <int K>
__device__ __forceinline__ uint4 basemul_row(const uint4 (&a)[K], const uint4 (&b)[K],
                                             const uint32_t (&zr)[4]) {
  uint32_t o[4];
#pragma unroll
  for (int u = 0; u < 4; u++) {
    int32_t t00 = 0, t11 = 0, t1 = 0;
#pragma unroll
    for (int j = 0; j < K; j++) {
      const uint32_t aw = u == 0 ? a[j].x : u == 1 ? a[j].y : u == 2 ? a[j].z : a[j].w;
      const uint32_t bw = u == 0 ? b[j].x : u == 1 ? b[j].y : u == 2 ? b[j].z : b[j].w;
      const int32_t a0 = (int16_t)(aw & 0xffffu), a1 = (int32_t)aw >> 16;
      const int32_t b0 = (int32_t)(bw & 0xffffu), b1 = (int32_t)(bw >> 16);  // [0, q)
      t00 += a0 * b0;
      t11 += a1 * b1;
      t1 += a0 * b1 + a1 * b0;
    }
    const uint32_t r00 = red_wide((uint32_t)t00 + kSumBias);  // [0, 3q)
    const uint32_t r11 = red_wide((uint32_t)t11 + kSumBias);
    const uint32_t r1 = red_wide((uint32_t)t1 + kSumBias);
    // r00 * 169 + r11 * zr < 3q * 169 + 3q * q < 2^31
    o[u] = pack2(red_wide(r00 * kRinv + r11 * zr[u]), red_wide(r1 * kRinv));
  }
  return make_uint4(o[0], o[1], o[2], o[3]);
}

// The same products with z folded into ntt(s) and 2^-16 left to the caller
// (the tiled kernel's inverse tables carry it).  zb = the lane's z_t * b1
// for its four pairs of one polynomial (b1 in [0, q)), as 16-bit values in
// [0, q + 4): red_wide of a product below q^2 is off by less than 0.002 q.
__device__ __forceinline__ uint2 pair_zb(const uint4 b, const uint32_t (&z)[4]) {
  const uint32_t p0 = red_wide((b.x >> 16) * z[0]), p1 = red_wide((b.y >> 16) * z[1]);
  const uint32_t p2 = red_wide((b.z >> 16) * z[2]), p3 = red_wide((b.w >> 16) * z[3]);
  return make_uint2(p0 | (p1 << 16), p2 | (p3 << 16));
}

constexpr uint32_t kSumBiasZ = 3329u << 19;  // >= |sum| (< 2^29.71); sum + bias < 2^32

// Per pair, out0 = sum_j a0 b0 + a1 (z b1), out1 = sum_j a0 b1 + a1 b0, each
// reduced once: 2^16 times the reference's basemul-accumulate, mod q.  With
// b0, b1 < q and z b1 < q + 4, |sum| <= 2K * 32768 * (q + 3) < 2^29.71 for
// K <= 4, so the biased sums lie in [0, 2^32) and red_wide leaves [0, 1.41 q).
template <int K>
__device__ __forceinline__ uint4 basemul_row_z(const uint4 (&a)[K], const uint4 (&b)[K],
                                               const uint2 (&zb)[K]) {
  uint32_t o[4];
#pragma unroll
  for (int u = 0; u < 4; u++) {
    uint32_t t0 = kSumBiasZ, t1 = kSumBiasZ;
#pragma unroll
    for (int j = 0; j < K; j++) {
      const uint32_t aw = u == 0 ? a[j].x : u == 1 ? a[j].y : u == 2 ? a[j].z : a[j].w;
      const uint32_t bw = u == 0 ? b[j].x : u == 1 ? b[j].y : u == 2 ? b[j].z : b[j].w;
      const uint32_t zw = u < 2 ? zb[j].x : zb[j].y;
      const int32_t a0 = (int16_t)(aw & 0xffffu), a1 = (int32_t)aw >> 16;
      const int32_t b0 = (int32_t)(bw & 0xffffu), b1 = (int32_t)(bw >> 16);
      const int32_t z1 = (int32_t)((u & 1) ? zw >> 16 : zw & 0xffffu);
      t0 += (uint32_t)(a0 * b0 + a1 * z1);
      t1 += (uint32_t)(a0 * b1 + a1 * b0);
    }
    o[u] = pack2(red_wide(t0), red_wide(t1));
  }
  return make_uint4(o[0], o[1], o[2], o[3]);
}

}  // namespace tk
