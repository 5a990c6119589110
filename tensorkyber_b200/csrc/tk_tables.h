// tk_tables.h -- constant tables of the matrix-form NTT and their layout contract.
//
// The ring is Z_3329[x]/(x^256+1).  A polynomial r[256] is viewed as a 16x16 grid
// r[16*m + c]: m is the "block" index (bits 4..7 of the coefficient index) and c
// the position inside a 16-coefficient block (bits 0..3).  TensorKyber's method
// (ntt_bench/ntt_kernels.cuh:140-148, 842-925) splits the 7-layer transform
// into two constant linear maps mod q:
//
//   forward   stage 1: layers 1-4 (len 128..16) act on m only:
//                      y[i][c]  = sum_m M1[i][m]      * x[m][c]
//             stage 2: layers 5-7 (len 8..2) act inside block i:
//                      z[i][c'] = sum_c M2[i][c'][c]  * y[i][c]
//   inverse   stage A: GS layers len 2..8 inside block m:
//                      y[m][c]  = sum_c' MA[m][c][c'] * x[m][c']
//             stage B: GS layers len 16..128 and the final x1441 Montgomery
//                      factor act on m:  z[i][c] = sum_m Minv[i][m] * y[m][c]
//
// The builder below derives all four by pushing unit vectors through a plain
// modular restatement of the layer code, exactly the probing construction of
// the reference's setup_tc_matrices (ntt_kernels.cuh:831-925).
//
// Device formulation (this build's own, see tk_ntt_mma.cu):
//   * Data enter the int8 tensor cores as raw BYTES (u8 operand).  A 16-bit
//     value v = b0 + 256*b1 contributes b0 and b1 on two K positions whose
//     constants are C and (256*C mod q), so no CUDA-core limb split of the
//     data is ever done.  Signed inputs are biased to unsigned first
//     (x ^ 0x8000 = x + 32768 with the row sum folded into the accumulator
//     init, or + 10q which is 0 mod q).
//   * Every constant is stored as two 7-bit INT8 limbs, lo in [0,127] and
//     hi in [0,26], on two accumulator groups g = 0, 1; the partial sums are
//     recombined as S = D_lo + 128 * D_hi with one IMAD.
//   * Stage-2 / stage-A matrices never mix even and odd c (len 8, 4, 2
//     butterflies keep the parity), so each is applied as two 8x8 halves.
#pragma once
#include <stdint.h>

namespace tk {

constexpr int kN = 256;
constexpr int kQ = 3329;

// floor(2^32 / q): lazy Barrett, S - umulhi(S, kBarLazy) * q in [0, q + 11)
// for S < 2^25, [0, q + 6) for S < 2^24.
constexpr uint32_t kBarLazy = 1290167u;
// ceil(2^38 / q): exact reduction floor(S / q) = umulhi(S, kBarExact) >> 6 for
// every 0 <= S < 2^26 (the error term S * e / 2^38 < 2^-12 < 1/q).
constexpr uint32_t kBarExact = 82570715u;

// Bias that makes a signed int16 an unsigned 16-bit value without changing it
// mod q: (x ^ 0x8000) + 522 = x + 33290 = x + 10q, valid for x <= 32245.
constexpr uint32_t kBias10qPacked = 0x020A020Au;

// ---- fragment tables (per lane, in the register order of mma.sync) -------
// Forward stage 1: A = 16x32 s8, rows i (output block), K k = 2*m + byte.
// Two accumulator groups (lo / hi limbs) -> two A fragments of 4 regs.
// c1: accumulator init of group 0 for rows (lane>>2) and (lane>>2)+8: the
// (-32768 * rowsum) mod q correction of the x ^ 0x8000 bias.
// Forward stage 2: per block b and parity s, A = 16x16 s8 (m16n8k16):
// rows r<8 -> group 0, r>=8 -> group 1, output c' = 2*(r&7) + s; K k = 2*slot
// + byte, slot j holds c = 2*e(j) + s with e(j) = (j>>1) + 4*(j&1).
// Forward stage 2 from int32 intermediates (s2w, the "wide" kernels): per
// block b and parity s, A = 16x32 s8 (m16n8k32); rows as s2; K k = 4*slot +
// byte, the four bytes of a non-negative 32-bit stage-1 sum S (< 2^25), whose
// byte j carries the constant times 256^j mod q; slot order as s2.
// Forward stage 1, single-limb form (inputs in [-128, 127], one byte each):
// A = 16x16 s8 (m16n8k16), rows i, K k' holds block m = pi(k') with
// pi(4t + j) = 2t + j (j < 2), 8 + 2t + (j - 2) (j >= 2) -- the m order in
// which the bytes sit in a lane's k32 B fragment (see tk_stages.cuh); the
// data byte is x + 128 (low byte xor 0x80) and c1b holds the
// (-128 * rowsum) mod q correction.
struct FwdFrags {
  uint32_t s1[2][32][4];
  int32_t c1[32][2];
  uint32_t s2[16][2][32][2];
  uint32_t s1b[2][32][2];
  int32_t c1b[32][2];
  uint32_t s2w[16][2][32][4];
};

// Inverse stage A: per block m and parity s, A = 16x16 s8; rows as in forward
// stage 2 (output c' = 2*(r&7) + s); K k = 2*slot + byte with the forward
// stage-2 slot order (slot j holds input c = 2*e(j) + s).  Inputs are biased
// with x ^ 0x8000; ca holds the group-0 accumulator init of row lane/4, the
// (-32768 * rowsum) mod q correction (the fused matrix-vector kernel's; the
// batch kernels cancel the bias in stage B instead, cbz below).
// Inverse stage B: A = 16x32 s8, rows i, K k = 2*m + byte; no correction (the
// kernels centre the output in the reduction, red_centred).
// Inverse stage B from int32 intermediates (sbw, the "wide" kernels): per limb
// g and K chunk j (blocks m = 8j .. 8j+7), A = 16x32 s8, rows i, K k =
// 4*(m - 8j) + byte, the four bytes of a non-negative stage-A sum (< 2^24),
// byte t carrying the constant times 256^t mod q; the two chunks accumulate
// into one accumulator.
// cbz: stage B's group-0 accumulator init when stage A runs without ca
// (the batch kernels): stage A's output then carries 32768 * rowsum(MA[m][c])
// mod q too, and stage B, linear, maps that to the constant Minv * offset;
// cbz[lane][t] = -(Minv * offset) mod q at the lane's D registers of n-tile t
// (rows lane/4 and lane/4 + 8, columns c = 8t + 2(lane%4) and c + 1).
struct InvFrags {
  uint32_t sa[16][2][32][2];
  int32_t ca[16][2][32];
  uint32_t sb[2][32][4];
  uint32_t sbw[2][2][32][4];
  int32_t cbz[32][2][4];
};

// Logical matrices (canonical residues in [0, q)).
struct Matrices {
  int16_t m1[16][16];        // [i][m]
  int16_t m2[16][16][16];    // [block][c'][c]
  int16_t ma[16][16][16];    // [block][c][c']  (output c, input c')
  int16_t minv[16][16];      // [i][m]
};

// Basemul pair constants: pair t (coefficients 2t, 2t+1) of the NTT domain
// is the residue mod X^2 - z_t, z_t = +-17^brv7(64 + t/2) (sign + for even t);
// zr[t] = z_t * 2^-16 mod q (the reference's basemul multiplies by 2^-16).
void build_pair_constants(int32_t zr[128]);
// z[t] = z_t itself, in [0, q).
void build_pair_roots(int32_t z[128]);

// Scales the inverse transform by f (mod q): Minv <- f * Minv, so that tables
// built from M compute f * invntt.
void scale_inverse(Matrices* M, int64_t f);

// B operands of the tcgen05 kernels (tk_tc5.cu), one 1 KiB tile per MMA
// shape: N = 32 rows (n = out + 16 * limb: output coefficient, 7-bit limb of
// the constant) x K = 32 bytes, int8 values, in the tcgen05 K-major layout
// without swizzle: row n, K byte k at (n / 8) * 256 + (k / 16) * 128 +
// (n % 8) * 16 + k % 16 (8-row core matrices of 16 bytes per row; the two
// K halves 128 bytes apart, 8-row groups 256 bytes apart).
//   tile 2m + t      inverse stage A (MA of block m): K byte k = 2 c' + b,
//                    byte b of input coefficient c'.  t = 0 (unsigned data):
//                    the low bytes, constant MA[m][out][c']; t = 1 (signed
//                    data): the high bytes, constant 256 MA[m][out][c'] mod
//                    q; the other byte's rows are zero.
//   tile 32 + h      inverse stage B (Minv), K step h: K byte k = 4 (m - 8h)
//                    + j, byte j of the non-negative (below 2^25) int32
//                    stage-A sum of block m; constant Minv[out][m] 256^j mod q.
//   tile 34 + t      forward stage 1 (M1): K byte k = 2 m + b, byte b of the
//                    block-m coefficient; t = 0: low bytes, constant
//                    M1[out][m]; t = 1: high bytes, 256 M1[out][m] mod q.
//   tile 36 + 2i + h forward stage 2 (M2 of block i), K step h: K byte k =
//                    4 (c - 8h) + j, byte j of the non-negative (below 2^25)
//                    int32 stage-1 sum of coefficient c; constant
//                    M2[i][out][c] 256^j mod q.
// The inverse uses tiles 0-33, the forward tiles 34-67.
constexpr int kTc5TileBytes = 1024;
constexpr int kTc5InvTiles = 34;
constexpr int kTc5FwdTiles = 34;
constexpr int kTc5Tiles = kTc5InvTiles + kTc5FwdTiles;
constexpr int kTc5TableBytes = kTc5Tiles * kTc5TileBytes;
inline int tc5_tile_offset(int n, int k) {
  return (n >> 3) * 256 + (k >> 4) * 128 + (n & 7) * 16 + (k & 15);
}
void build_tc5_tables(const Matrices& M, uint8_t* out /* kTc5TableBytes */);

void build_matrices(Matrices* M);
void build_fwd_frags(const Matrices& M, FwdFrags* F);
void build_inv_frags(const Matrices& M, InvFrags* F);

// Slot order inside a forward stage-2 parity half.
inline int fwd_slot_e(int slot) { return (slot >> 1) + 4 * (slot & 1); }
// Block m of single-limb stage-1 K position k (FwdFrags::s1b).
int basic_k_block(int k);

}  // namespace tk
