// tk_ntt_mma.cu -- batched ML-KEM NTT / iNTT on sm_100a: tensor-TMA staging +
// int8 mma.sync tiles, CTA-cooperative persistent tiles.
//
// A CTA of W warps owns a ring of S shared-memory slots; each slot holds a
// tile of 8*W polynomials in padded 528-byte rows (the 16-byte pad makes the
// block-wise accesses below bank-conflict free).  The pad comes from the TMA
// box itself: the global batch is described as a [npoly][128] uint32 tensor
// and every copy moves a box of 8 rows x 132 words, whose last 4 words per row
// are out of bounds (zero-filled on load, skipped on store); polynomials past
// npoly are out of bounds the same way, so ragged tails need no special code.
// CTA c owns the contiguous run of 8-polynomial units
// [c*U/G, (c+1)*U/G) (U units, G CTAs), so CTAs differ by at most one unit of
// work; it walks that run in tiles of W units (a warp whose unit lies past
// the run issues no copy).  Launches use programmatic dependent launch: the
// prologue (constants to registers, mbarrier set-up) overlaps the tail of the
// previous kernel in the stream and griddepcontrol.wait precedes the first
// global access.  Per tile:
//
//   load     lane 0 of warp w: mbarrier.arrive.expect_tx + one tensor TMA for
//            polynomials 8w .. 8w+7 of the tile
//   forward  stage 1 (M1, layers 1-4), by polynomial: warp w, polys 8w..8w+7:
//              ldmatrix.trans -> 4 x mma m16n8k32 s8.u8 -> S = D_lo + 128 D_hi
//              -> lazy Barrett -> parity-split rows, in place
//            CTA barrier
//            stage 2 (M2, layers 5-7), by block: warp w, blocks (16/W)w ..:
//              ldmatrix -> 4 x mma m16n8k16 -> exact Barrett to [0, q)
//              -> natural order, in place
//            CTA barrier, then lane 0 of warp w stores polys 8w .. 8w+7
//   inverse  stage A (MA) by block (as forward stage 2, lazy Barrett, natural
//            order), CTA barrier, stage B (Minv) by polynomial (as forward
//            stage 1, output centred), then each warp stores its own polys
//   store    tensor TMA smem -> global; at the top of the next iteration the
//            slot is refilled (S-1 tiles ahead, S = slots) once that store was
//            read out of smem (wait_group.read), so S-1 loads stay in flight
//            while a tile is computed
//
// Wide kernels (kWide): the first stage's sums are not reduced mod q; they go
// as int32 to a tile of 1040-byte rows after the slots, and the second stage
// reads their four bytes with m16n8k32 MMAs whose constants carry the byte
// weights 256^j mod q.  Forward: stage 1 writes the tile by polynomial, stage
// 2 reads it by block (the same MMA count as the k16 form).  Inverse: stage A
// writes it by block in [c][m] order, stage B reads it by polynomial (two K
// chunks, twice the MMAs).
//
// Reference counterparts: the in-place batch kernels k_ntt_2tc_tc_cc /
// k_invntt_2tc_tc_cc / k_ntt_tc_cc_cp / k_invntt_tc_cc_cp
// (ntt_bench/ntt_bench.cu:61-131, 181-277) over ntt_core / intt_core
// (ntt_bench/ntt_kernels.cuh:393-489, 548-625).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <mutex>
#include <type_traits>

#include "tk_internal.h"
#include "tk_ptx.cuh"
#include "tk_stages.cuh"
#include "tk_tables.h"

namespace tk {

constexpr int kWarpBoxBytes = 8 * kRowBytes;      // one TMA box: 8 padded rows
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // every mbarrier wait gives up after 2 s

__device__ FwdFrags g_fwd;
__device__ InvFrags g_inv;
__device__ unsigned int g_status;

// Kernel parameters.  OneSeg: one batch (every launch but the multi-batch
// ones), its tensor maps at fixed offsets.  SegMaps: up to kMaxSegs
// independent batches ("segments") in one launch.  Units (8 polynomials) are numbered across segments: segment j owns
// units [first_unit[j], first_unit[j+1]); its rows are addressed through its
// own tensor maps (in, out) and, for the inverse with addend, its own addend
// (npoly[j] polynomials).
struct OneSeg {
  CUtensorMap in;
  CUtensorMap out;
  const uint32_t* addend;
  int npoly;
};
struct SegMaps {
  CUtensorMap in[kMaxSegs];
  CUtensorMap out[kMaxSegs];
  const uint32_t* addend[kMaxSegs];
  int npoly[kMaxSegs];
  int first_unit[kMaxSegs + 1];
  int nseg;
};

// Forward input forms: int16 polynomials (any value), int16 polynomials with
// coefficients in [-128, 127] (single-limb stage 1), and packed 2- or 3-bit
// fields (TC-PACK format, single-limb stage 1).
enum InForm { kInInt16 = 0, kInSmall = 1, kInPack2 = 2, kInPack3 = 3 };
template <int kIn>
constexpr int packed_row_bytes() {
  return kIn == kInPack2 ? 64 : kIn == kInPack3 ? 128 : 0;
}

template <int W, int S, int kIn = kInInt16, bool kWide = false>
struct Cfg {
  static constexpr int kWarps = W;
  static constexpr int kThreads = 32 * W;
  static constexpr int kTile = 8 * W;                 // polynomials per tile
  // a slot: kTile padded rows, then (packed forms) the tile's packed input
  static constexpr int kPackBytes = packed_row_bytes<kIn>();
  static constexpr int kRowsBytes = kTile * kRowBytes;
  static constexpr int kSlotBytes = kTile * (kRowBytes + kPackBytes);
  static constexpr int kSlots = S;
  // wide kernels: one tile of int32 stage-1 sums after the slots
  static constexpr int kInterBytes = kWide ? kTile * kWideRowBytes : 0;
  static constexpr int kSmem = S * kSlotBytes + kInterBytes + 16 * S;  // + mbarriers
  static constexpr int kBlocksPerWarp = 16 / W;       // block-wise stages
  static constexpr int kPairsPerWarp = kBlocksPerWarp / 2;
  // CTAs per SM the shared memory allows; also the register cap for ptxas
  static constexpr int kMinBlocks = (227 * 1024) / (kSmem + 1024);
  static_assert(W == 4 || W == 8, "4 or 8 warps per CTA");
};

__device__ __forceinline__ void cta_sync_named() {
  asm volatile("bar.sync 1;" ::: "memory");
}

// Block-wise stage of one tile for this warp: P block pairs x NT n-tiles of 8
// polynomials (NT = W: a full tile), the next unit's ldmatrix issued ahead of
// the current stores.  Inverse input is biased (x ^ 0x8000) and parity-split
// here; forward input is already parity-split by stage 1.
template <bool kInverse, int W, int P, int NT = W>
__device__ __forceinline__ void block_stage(uint32_t slot, uint8_t* slotp, int blk0,
                                            uint32_t ldc_off, uint32_t stc_off,
                                            const uint32_t (&ac)[P][2][2][2],
                                            const int32_t (&cc)[P][2][2]) {
  constexpr int kIters = P * NT;
  uint32_t r[4];
  ldsm_x4(slot + 32u * blk0 + ldc_off, r[0], r[1], r[2], r[3]);
#pragma unroll
  for (int it = 0; it < kIters; it++) {
    const int p = it / NT, nt = it % NT;
    uint32_t n[4] = {0, 0, 0, 0};
    if (it + 1 < kIters) {
      const int p1 = (it + 1) / NT, nt1 = (it + 1) % NT;
      ldsm_x4(slot + nt1 * 8 * kRowBytes + 32u * (blk0 + 2 * p1) + ldc_off, n[0], n[1], n[2],
              n[3]);
    }
    uint32_t x[4];
    if (kInverse) {
      // r = (I: c 2q,2q+1 | I: c 8+2q,9+2q | I+1: ...); bias, then parity split
      // into slots (c=2q | c=8+2q) and (c=2q+1 | c=9+2q)
      const uint32_t x0 = r[0] ^ 0x80008000u, x1 = r[1] ^ 0x80008000u;
      const uint32_t x2 = r[2] ^ 0x80008000u, x3 = r[3] ^ 0x80008000u;
      x[0] = __byte_perm(x0, x1, 0x5410);
      x[1] = __byte_perm(x0, x1, 0x7632);
      x[2] = __byte_perm(x2, x3, 0x5410);
      x[3] = __byte_perm(x2, x3, 0x7632);
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) x[j] = r[j];
    }
    stage_c<kInverse>(ac[p], cc[p], x,
                      slotp + nt * 8 * kRowBytes + 32 * (blk0 + 2 * p) + stc_off);
#pragma unroll
    for (int j = 0; j < 4; j++) r[j] = n[j];
  }
}

// Forward stage 2 from the tile's int32 intermediates (wide kernels): as
// block_stage, two ldmatrix.x4 per block pair (one per block).  ldw[p]: this
// lane's ldmatrix row offset of pair p's first block (polynomial lane&7 of
// the n-tile, parity (lane/16) placed by the row swizzle, half (lane/8)&1).
template <int W, int P>
__device__ __forceinline__ void block_stage_wide(uint32_t inter, uint8_t* slotp, int blk0,
                                                 const uint32_t (&ldw)[P], uint32_t stc_off,
                                                 const uint32_t (&ac)[P][2][2][4]) {
  constexpr int kIters = P * W;
  uint32_t r[8];
  ldsm_x4(inter + ldw[0], r[0], r[1], r[2], r[3]);
  ldsm_x4(inter + ldw[0] + 64, r[4], r[5], r[6], r[7]);
#pragma unroll
  for (int it = 0; it < kIters; it++) {
    const int p = it / W, nt = it % W;
    uint32_t n[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (it + 1 < kIters) {
      const int p1 = (it + 1) / W, nt1 = (it + 1) % W;
      const uint32_t a1 = inter + nt1 * 8 * kWideRowBytes + ldw[p1];
      ldsm_x4(a1, n[0], n[1], n[2], n[3]);
      ldsm_x4(a1 + 64, n[4], n[5], n[6], n[7]);
    }
    stage_c_wide(ac[p], r, slotp + nt * 8 * kRowBytes + 32 * (blk0 + 2 * p) + stc_off);
#pragma unroll
    for (int j = 0; j < 8; j++) r[j] = n[j];
  }
}

// Inverse stage A of one tile into the int32 intermediates (wide kernels): as
// block_stage<true>, the sums of pair p stored at offsets ia[p][s] of the rows
// of polynomials 2q, 2q+1 of each n-tile.
template <int W, int P>
__device__ __forceinline__ void block_stage_inv_wide(uint32_t slot, int blk0, uint32_t ldc_off,
                                                     uint8_t* interp, uint32_t row_off,
                                                     const uint32_t (&ia)[P][2],
                                                     const uint32_t (&ac)[P][2][2][2],
                                                     const int32_t (&cc)[P][2][2]) {
  constexpr int kIters = P * W;
  uint32_t r[4];
  ldsm_x4(slot + 32u * blk0 + ldc_off, r[0], r[1], r[2], r[3]);
#pragma unroll
  for (int it = 0; it < kIters; it++) {
    const int p = it / W, nt = it % W;
    uint32_t n[4] = {0, 0, 0, 0};
    if (it + 1 < kIters) {
      const int p1 = (it + 1) / W, nt1 = (it + 1) % W;
      ldsm_x4(slot + nt1 * 8 * kRowBytes + 32u * (blk0 + 2 * p1) + ldc_off, n[0], n[1], n[2],
              n[3]);
    }
    const uint32_t x0 = r[0] ^ 0x80008000u, x1 = r[1] ^ 0x80008000u;
    const uint32_t x2 = r[2] ^ 0x80008000u, x3 = r[3] ^ 0x80008000u;
    const uint32_t x[4] = {__byte_perm(x0, x1, 0x5410), __byte_perm(x0, x1, 0x7632),
                           __byte_perm(x2, x3, 0x5410), __byte_perm(x2, x3, 0x7632)};
    stage_c_inv_wide(ac[p], cc[p], x, interp + nt * 8 * kWideRowBytes + row_off, ia[p]);
#pragma unroll
    for (int j = 0; j < 4; j++) r[j] = n[j];
  }
}

// Inverse stage B of this warp's 8 polynomials from the int32 intermediates
// (wide kernels; irow0: the first one's row), two ldmatrix.x4 per polynomial,
// the next one's issued ahead; addend as poly_stage.
template <bool kAdd>
__device__ __forceinline__ void poly_stage_inv_wide(uint32_t irow0, uint8_t* minep,
                                                    const uint32_t (&lb)[2],
                                                    const uint32_t (&a)[2][2][4],
                                                    const int32_t (&cb)[2][4], uint32_t w_nat,
                                                    const uint32_t* addend, int poly0, int npoly,
                                                    uint32_t add_off) {
  auto load_add = [&](int p, uint32_t (&e)[4]) {
    const int poly = poly0 + p;
    if (kAdd && addend != nullptr && poly < npoly) {
      const uint32_t* w = addend + (size_t)poly * 128 + add_off;
      e[0] = __ldg(w);
      e[1] = __ldg(w + 4);
      e[2] = __ldg(w + 64);
      e[3] = __ldg(w + 68);
    } else {
      e[0] = e[1] = e[2] = e[3] = 0;
    }
  };
  uint32_t b[2][4], e[4];
  ldsm_x4(irow0 + lb[0], b[0][0], b[0][1], b[0][2], b[0][3]);
  ldsm_x4(irow0 + lb[1], b[1][0], b[1][1], b[1][2], b[1][3]);
  load_add(0, e);
#pragma unroll
  for (int p = 0; p < 8; p++) {
    uint32_t n[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, en[4] = {0, 0, 0, 0};
    if (p < 7) {
      const uint32_t nx = irow0 + (p + 1) * kWideRowBytes;
      ldsm_x4(nx + lb[0], n[0][0], n[0][1], n[0][2], n[0][3]);
      ldsm_x4(nx + lb[1], n[1][0], n[1][1], n[1][2], n[1][3]);
      load_add(p + 1, en);
    }
    stage_m_inv_wide<kAdd>(a, cb, b, minep + p * kRowBytes, w_nat, e);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      b[0][j] = n[0][j];
      b[1][j] = n[1][j];
      e[j] = en[j];
    }
  }
}

// Stage over m for this warp's 8 polynomials, the next ldmatrix issued ahead.
// Inverse with kAdd only: polynomial p of this warp (global index poly0 + p)
// gets addend[poly0 + p] added to its output; the addend words for
// polynomial p+1 are fetched while p is computed.
template <bool kInverse, bool kAdd = false>
__device__ __forceinline__ void poly_stage(uint32_t mine, uint8_t* minep, uint32_t ldt_off,
                                           const uint32_t (&am)[2][4], int32_t cm_lo,
                                           int32_t cm_hi, const int32_t (&cb)[2][4],
                                           uint32_t w_even, uint32_t w_odd,
                                           uint32_t w_nat, const uint32_t* addend, int poly0,
                                           int npoly, uint32_t add_off) {
  auto load_add = [&](int p, uint32_t (&e)[4]) {
    const int poly = poly0 + p;
    if (kInverse && kAdd && addend != nullptr && poly < npoly) {
      const uint32_t* w = addend + (size_t)poly * 128 + add_off;
      e[0] = __ldg(w);
      e[1] = __ldg(w + 4);
      e[2] = __ldg(w + 64);
      e[3] = __ldg(w + 68);
    } else {
      e[0] = e[1] = e[2] = e[3] = 0;
    }
  };
  uint32_t b[4], e[4];
  ldsm_x4_t(mine + ldt_off, b[0], b[1], b[2], b[3]);
  load_add(0, e);
#pragma unroll
  for (int p = 0; p < 8; p++) {
    uint32_t n[4] = {0, 0, 0, 0}, en[4] = {0, 0, 0, 0};
    if (p < 7) {
      ldsm_x4_t(mine + (p + 1) * kRowBytes + ldt_off, n[0], n[1], n[2], n[3]);
      load_add(p + 1, en);
    }
    if (kInverse)
      stage_m_q<true, kAdd>(am, cb[0], cb[1], b[0], b[1], b[2], b[3], minep + p * kRowBytes, 0, 0,
                    w_nat, e);
    else  // x ^ 0x8000 bias; the 32768 * rowsum term is cancelled by cm_lo/cm_hi
      stage_m<false>(am, cm_lo, cm_hi, b[0] ^ 0x80008000u, b[1] ^ 0x80008000u,
                     b[2] ^ 0x80008000u, b[3] ^ 0x80008000u, minep + p * kRowBytes, w_even,
                     w_odd, 0, e);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      b[j] = n[j];
      e[j] = en[j];
    }
  }
}

// Forward stage 1 of this warp's 8 polynomials in single-limb form.  kInSmall:
// operands from the int16 rows (ldmatrix.trans as poly_stage, low bytes);
// packed forms: from the tile's packed rows (packp: this warp's 8 rows of
// kPackBytes), which lane (t = lane%4, n = lane/4) reads as the words of blocks
// m = 2t, 2t+1, 8+2t, 9+2t.  Output to minep's rows (kRowBytes apart,
// parity-split int16), or with kWideOut unreduced to int32 intermediate rows
// (kWideRowBytes apart; w_even / w_odd then the wide offsets).
template <int kIn, bool kWideOut = false>
__device__ __forceinline__ void poly_stage_small(uint32_t mine, uint8_t* minep, uint32_t ldt_off,
                                                 const uint8_t* packp, const uint32_t (&ab)[2][2],
                                                 int32_t cb_lo, int32_t cb_hi, uint32_t w_even,
                                                 uint32_t w_odd, int lane, uint32_t* bad) {
  constexpr int kOutRow = kWideOut ? kWideRowBytes : kRowBytes;
  auto out = [&](int p, uint32_t bt0, uint32_t bt1) {
    if constexpr (kWideOut)
      stage_m_small_wide(ab, cb_lo, cb_hi, bt0, bt1, minep + p * kOutRow, w_even, w_odd);
    else
      stage_m_small(ab, cb_lo, cb_hi, bt0, bt1, minep + p * kOutRow, w_even, w_odd);
  };
  const uint32_t t = lane & 3, n = lane >> 2;
  if (kIn == kInSmall) {
    uint32_t b[4];
    ldsm_x4_t(mine + ldt_off, b[0], b[1], b[2], b[3]);
#pragma unroll
    for (int p = 0; p < 8; p++) {
      uint32_t nx[4] = {0, 0, 0, 0};
      if (p < 7) ldsm_x4_t(mine + (p + 1) * kRowBytes + ldt_off, nx[0], nx[1], nx[2], nx[3]);
      const uint32_t bt0 = small_operand(b[0], b[1], bad);
      const uint32_t bt1 = small_operand(b[2], b[3], bad);
      out(p, bt0, bt1);
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = nx[j];
    }
  } else if (kIn == kInPack2) {
    // 4 bytes per block m (coefficients 16m .. 16m+15); coefficient c of the
    // block is byte c/4, bits 2(c%4): n-tile 0 byte n/4, n-tile 1 byte 2 + n/4
    const uint32_t k0 = n >> 2, k1 = k0 + 2;
    const uint32_t sel0 = k0 | ((k0 + 4) << 4), sel1 = k1 | ((k1 + 4) << 4);
    const uint32_t shift = 2 * (n & 3);
#pragma unroll
    for (int p = 0; p < 8; p++) {
      const uint8_t* pk = packp + p * 64;
      const uint2 v01 = *(const uint2*)(pk + 8 * t);       // m = 2t, 2t+1
      const uint2 v23 = *(const uint2*)(pk + 32 + 8 * t);  // m = 8+2t, 9+2t
      const uint32_t bt0 = packed_operand<2>(v01.x, v01.y, v23.x, v23.y, sel0, shift);
      const uint32_t bt1 = packed_operand<2>(v01.x, v01.y, v23.x, v23.y, sel1, shift);
      out(p, bt0, bt1);
    }
  } else {
    // 8 bytes per block m; coefficient c is byte c/2, bits 3(c%2): n-tile 0
    // uses each block's first word (byte n/2), n-tile 1 its second word
    const uint32_t k = n >> 1;
    const uint32_t sel = k | ((k + 4) << 4);
    const uint32_t shift = 3 * (n & 1);
#pragma unroll
    for (int p = 0; p < 8; p++) {
      const uint8_t* pk = packp + p * 128;
      const uint4 v01 = *(const uint4*)(pk + 16 * t);       // m = 2t, 2t+1
      const uint4 v23 = *(const uint4*)(pk + 64 + 16 * t);  // m = 8+2t, 9+2t
      const uint32_t bt0 = packed_operand<3>(v01.x, v01.z, v23.x, v23.z, sel, shift);
      const uint32_t bt1 = packed_operand<3>(v01.y, v01.w, v23.y, v23.w, sel, shift);
      out(p, bt0, bt1);
    }
  }
}

// ------------------------------------------------------------ the kernel ---
template <bool kInverse, int W, int S, int kIn = kInInt16, bool kAdd = false,
          class Param = OneSeg, bool kWide = false>
__global__ void __launch_bounds__(32 * W, Cfg<W, S, kIn, kWide>::kMinBlocks)
    k_ntt_mma(const __grid_constant__ Param segs) {
  constexpr bool kMulti = std::is_same<Param, SegMaps>::value;
  static_assert(!kInverse || kIn == kInInt16, "input forms are forward only");
  static_assert(kInverse || !kAdd, "the addend is an inverse option");
  static_assert(!kWide || ((kIn == kInInt16 || !kInverse) && !(kMulti && kInverse)),
                "wide: the inverse with int16 input and one segment");
  using C = Cfg<W, S, kIn, kWide>;
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  int nunits;
  if constexpr (kMulti)
    nunits = segs.first_unit[segs.nseg];
  else
    nunits = (segs.npoly + 7) >> 3;
  const int u_begin = (int)((long long)blockIdx.x * nunits / gridDim.x);
  const int u_end = (int)((long long)(blockIdx.x + 1) * nunits / gridDim.x);
  const int nmine = (u_end - u_begin + W - 1) / W;  // tiles of this CTA (CTA-uniform)

  const uint32_t smem0 = smem_u32(smem);
  const uint32_t inter = smem0 + C::kSlots * C::kSlotBytes;  // wide: int32 intermediates
  uint8_t* const interp = smem + C::kSlots * C::kSlotBytes;
  const uint32_t bar0 = inter + C::kInterBytes;

  // ---- constants of this warp's role -> registers -------------------------
  uint32_t am[2][4];                       // stage over m (fwd M1 / inv Minv)
  int32_t cm_lo, cm_hi;                    // its accumulator init
  constexpr int kAW = kWide && !kInverse ? 4 : 2;  // A registers (k16, or k32 wide forward)
  uint32_t ac[C::kPairsPerWarp][2][2][kAW];  // block-wise stage, per (pair, block, parity)
  // block-wise stage accumulator init: zero (the inverse's stage-A bias
  // offset is cancelled by stage B's init cb instead)
  int32_t cc[C::kPairsPerWarp][2][2];
  int32_t cb[2][4];  // inverse stage B: group-0 init per n-tile (InvFrags::cbz)
#pragma unroll
  for (int t = 0; t < 2; t++)
#pragma unroll
    for (int j = 0; j < 4; j++) cb[t][j] = kInverse ? g_inv.cbz[lane][t][j] : 0;
  const int blk0 = C::kBlocksPerWarp * warp;
#pragma unroll
  for (int g = 0; g < 2; g++)
#pragma unroll
    for (int j = 0; j < 4; j++) am[g][j] = kInverse ? g_inv.sb[g][lane][j] : g_fwd.s1[g][lane][j];
  uint32_t amw[2][2][4];  // wide inverse stage B: [limb][K chunk]
  if constexpr (kWide && kInverse) {
#pragma unroll
    for (int g = 0; g < 2; g++)
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j = 0; j < 4; j++) amw[g][c][j] = g_inv.sbw[g][c][lane][j];
  }
  cm_lo = kInverse ? 0 : g_fwd.c1[lane][0];
  cm_hi = kInverse ? 0 : g_fwd.c1[lane][1];
  uint32_t ab[2][2] = {{0, 0}, {0, 0}};  // single-limb stage 1 (input forms)
  int32_t cb_lo = 0, cb_hi = 0;
  if (kIn != kInInt16) {
#pragma unroll
    for (int g = 0; g < 2; g++)
#pragma unroll
      for (int j = 0; j < 2; j++) ab[g][j] = g_fwd.s1b[g][lane][j];
    cb_lo = g_fwd.c1b[lane][0];
    cb_hi = g_fwd.c1b[lane][1];
  }
  uint32_t bad = 0;  // kInSmall: inputs outside [-128, 127] seen
#pragma unroll
  for (int p = 0; p < C::kPairsPerWarp; p++)
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int b = blk0 + 2 * p + h;
#pragma unroll
        for (int j = 0; j < kAW; j++)
          ac[p][h][s][j] = (kWide && !kInverse) ? g_fwd.s2w[b][s][lane][j]
                           : kInverse ? g_inv.sa[b][s][lane][j & 1]
                                      : g_fwd.s2[b][s][lane][j & 1];
        cc[p][h][s] = 0;
      }

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < C::kSlots; s++) mbar_init(bar0 + 8 * s, W);
    fence_mbar_init();
  }
  __syncthreads();
  // Everything above overlaps the previous kernel in the stream; from here on
  // global memory that it may have written is read.
  grid_dependency_wait();
  grid_launch_dependents();
  if (nmine == 0) return;  // CTA-uniform

  const int q4 = lane & 3, g8 = lane >> 2;
  // ldmatrix.trans rows of the stage over m: matrix j = lane/8 covers
  // m = (lane&7) + 8*(j&1), coefficients 8*(j>>1) .. +7.  The inverse's
  // intermediate (stage A's output) keeps the two 16-byte coefficient halves
  // of block m swapped when bit 2 of m is set, so that the eight rows of each
  // matrix (m = 0..7 or 8..15, 32 bytes apart) fall on eight different bank
  // groups instead of two rows per group.
  const uint32_t ldt_off = 32u * ((lane & 7) + 8 * ((lane >> 3) & 1)) +
                           16u * ((lane >> 4) ^ (kInverse ? (lane >> 2) & 1 : 0));
  // forward stage-1 stores: block i = lane/4 (and +8); the parity halves are
  // swapped in blocks with bit 2 set (bank spread).
  const uint32_t hb1 = (lane >> 4) & 1;
  const uint32_t w_even = 32u * g8 + 16u * hb1 + 4u * q4;
  const uint32_t w_odd = 32u * g8 + 16u * (hb1 ^ 1) + 4u * q4;
  const uint32_t w_nat = 32u * g8 + 4u * q4;  // inverse stage-B stores
  // block-wise stage: ldmatrix row = polynomial lane&7 of the n-tile, block
  // (pair base) + lane/16; forward reads the parity halves (lane/8)&1 xor the
  // block's bit 2 (uniform within a pair), inverse reads coefficient halves.
  const uint32_t hbw = (uint32_t)((blk0 >> 2) & 1);
  const uint32_t ldc_off = kRowBytes * (lane & 7) + 32u * (lane >> 4) +
                           16u * (kInverse ? ((lane >> 3) & 1) : (((lane >> 3) & 1) ^ hbw));
  // block-wise stage output: coefficient pair lane/4 of polynomials 2q, 2q+1;
  // the inverse's (the intermediate) with the halves swapped in blocks with
  // bit 2 set (the warp's blocks share that bit: hbw)
  const uint32_t stc_off = kRowBytes * (2 * q4) + 4u * (g8 ^ (kInverse ? 4 * hbw : 0));
  // wide kernels: stage-1 stores of block lane/4 (even / odd half, swizzled),
  // and the stage-2 ldmatrix rows of each block pair
  const uint32_t swz1 = (uint32_t)(g8 >> 1) & 1u;
  const uint32_t wi_e = 64u * g8 + 32u * swz1 + 8u * q4;
  const uint32_t wi_o = 64u * g8 + 32u * (swz1 ^ 1u) + 8u * q4;
  uint32_t ldw[C::kPairsPerWarp];
#pragma unroll
  for (int p = 0; p < C::kPairsPerWarp; p++) {
    const int I = blk0 + 2 * p;
    const uint32_t par = ((uint32_t)(lane >> 4) & 1u) ^ ((uint32_t)(I >> 1) & 1u);
    ldw[p] = kWideRowBytes * (lane & 7) + 64u * I + 32u * par + 16u * ((lane >> 3) & 1);
  }
  // wide inverse: stage-A stores (rows of polynomials 2q, 2q+1; c' = 2(lane/4)
  // + s; blocks I, I+1 side by side) and stage-B ldmatrix rows (n-tile t: row
  // c = 8t + lane%8, 16-byte chunk lane/8 under the row swizzle)
  const uint32_t ia_row = kWideRowBytes * (2u * q4);
  uint32_t ia[C::kPairsPerWarp][2];
#pragma unroll
  for (int p = 0; p < C::kPairsPerWarp; p++) {
    const uint32_t I = (uint32_t)(blk0 + 2 * p);
#pragma unroll
    for (int s = 0; s < 2; s++)
      ia[p][s] = 64u * (2 * g8 + s) + 16u * ((I >> 2) ^ ((uint32_t)g8 & 3u)) + 4u * (I & 3u);
  }
  uint32_t lb[2];
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const uint32_t r = (uint32_t)lane & 7u;
    lb[t] = 64u * (8 * t + r) + 16u * (((uint32_t)lane >> 3) ^ (r >> 1));
  }

  // ---- TMA issue: lane 0 of each warp moves its 8 polynomials (one box) ----
  // segment of a unit (units are numbered across the launch's segments), its
  // first unit, and its tensor maps, addend and size
  auto seg_of = [&](int unit) -> int {
    if constexpr (kMulti) {
      int sg = 0;
#pragma unroll
      for (int j = 1; j < kMaxSegs; j++) sg += (j < segs.nseg && unit >= segs.first_unit[j]);
      return sg;
    } else {
      return 0;
    }
  };
  auto seg_first = [&](int sg) -> int {
    if constexpr (kMulti) return segs.first_unit[sg]; else return 0;
  };
  auto map_in = [&](int sg) -> const CUtensorMap* {
    if constexpr (kMulti) return &segs.in[sg]; else return &segs.in;
  };
  auto map_out = [&](int sg) -> const CUtensorMap* {
    if constexpr (kMulti) return &segs.out[sg]; else return &segs.out;
  };
  auto seg_addend = [&](int sg) -> const uint32_t* {
    if constexpr (kMulti) return segs.addend[sg]; else return segs.addend;
  };
  auto seg_npoly = [&](int sg) -> int {
    if constexpr (kMulti) return segs.npoly[sg]; else return segs.npoly;
  };
  auto issue_load = [&](int k, int slot_i) {
    if (lane != 0) return;
    const int unit = u_begin + k * W + warp;
    const uint32_t bar = bar0 + 8 * slot_i;
    if (unit < u_end) {
      const int sg = seg_of(unit);
      const CUtensorMap* tm_in = map_in(sg);
      const int row = 8 * (unit - seg_first(sg));
      if (C::kPackBytes) {  // the packed rows, after the tile's padded rows
        mbar_expect_tx(bar, 8 * C::kPackBytes);
        tma_load_2d(smem0 + slot_i * C::kSlotBytes + C::kRowsBytes + warp * 8 * C::kPackBytes,
                    tm_in, 0, row, bar);
      } else {
        mbar_expect_tx(bar, kWarpBoxBytes);
        tma_load_2d(smem0 + slot_i * C::kSlotBytes + warp * kWarpBoxBytes, tm_in, 0, row, bar);
      }
    } else {
      mbar_expect_tx(bar, 0);  // arrive only
    }
  };
  auto issue_store = [&](int k, int slot_i) {
    if (lane != 0) return;
    const int unit = u_begin + k * W + warp;
    if (unit < u_end) {
      const int sg = seg_of(unit);
      tma_store_2d(map_out(sg), 0, 8 * (unit - seg_first(sg)),
                   smem0 + slot_i * C::kSlotBytes + warp * kWarpBoxBytes);
    }
    bulk_commit();
  };

  // prologue: tiles 0 .. S-2 into slots 0 .. S-2
#pragma unroll
  for (int t = 0; t < C::kSlots - 1; t++)
    if (t < nmine) issue_load(t, t);

  int slot_i = 0;
  uint32_t phase = 0;
  for (int k = 0; k < nmine; k++) {
    const uint32_t slot = smem0 + slot_i * C::kSlotBytes;
    uint8_t* slotp = smem + slot_i * C::kSlotBytes;
    const bool ok = mbar_wait_bounded(bar0 + 8 * slot_i, phase, kWaitLimitNs);
    if (!__syncthreads_and(ok)) {  // CTA-uniform give-up
      if (tid == 0) atomicOr(&g_status, kInverse ? 2u : 1u);
      break;
    }
    if (k + C::kSlots - 1 < nmine) {
      // refill early: tile k+S-1 goes to the slot that held tile k-1, whose
      // compute finished before the barrier above; its store (issued by this
      // lane, for this warp's rows) must have been read out of smem.
      if (lane == 0) bulk_wait_read<0>();
      int s2 = slot_i + C::kSlots - 1;
      if (s2 >= C::kSlots) s2 -= C::kSlots;
      issue_load(k + C::kSlots - 1, s2);
    }
    // own polynomials of this warp: rows 8w .. 8w+7
    const uint32_t mine = slot + 8 * warp * kRowBytes;
    uint8_t* minep = slotp + 8 * warp * kRowBytes;

    if constexpr (kWide && kInverse) {
      block_stage_inv_wide<W>(slot, blk0, ldc_off, interp, ia_row, ia, ac, cc);
      cta_sync_named();
      const int unit = u_begin + k * W + warp;
      poly_stage_inv_wide<kAdd>(inter + 8 * warp * kWideRowBytes, minep, lb, amw, cb,
                                w_nat, kAdd ? seg_addend(0) : nullptr, 8 * unit,
                                kAdd ? seg_npoly(0) : 0, 8u * g8 + q4);
      fence_proxy_async_smem();
      __syncwarp();
      issue_store(k, slot_i);
    } else if constexpr (kWide) {
      uint8_t* irow0 = interp + 8 * warp * kWideRowBytes;
      if constexpr (kIn == kInInt16) {
        uint32_t b[4];
        ldsm_x4_t(mine + ldt_off, b[0], b[1], b[2], b[3]);
#pragma unroll
        for (int p = 0; p < 8; p++) {
          uint32_t n[4] = {0, 0, 0, 0};
          if (p < 7) ldsm_x4_t(mine + (p + 1) * kRowBytes + ldt_off, n[0], n[1], n[2], n[3]);
          stage_m_wide(am, cm_lo, cm_hi, b[0] ^ 0x80008000u, b[1] ^ 0x80008000u,
                       b[2] ^ 0x80008000u, b[3] ^ 0x80008000u, irow0 + p * kWideRowBytes, wi_e,
                       wi_o);
#pragma unroll
          for (int j = 0; j < 4; j++) b[j] = n[j];
        }
      } else {
        uint32_t tile_bad = 0;  // as below: only live rows count
        poly_stage_small<kIn, true>(mine, irow0, ldt_off,
                                    slotp + C::kRowsBytes + warp * 8 * C::kPackBytes, ab, cb_lo,
                                    cb_hi, wi_e, wi_o, lane, &tile_bad);
        if (u_begin + k * W + warp < u_end) bad |= tile_bad;
      }
      cta_sync_named();
      block_stage_wide<W>(inter, slotp, blk0, ldw, stc_off, ac);
      fence_proxy_async_smem();
      cta_sync_named();
      issue_store(k, slot_i);
    } else if (!kInverse) {
      if (kIn == kInInt16)
        poly_stage<false>(mine, minep, ldt_off, am, cm_lo, cm_hi, cb, w_even, w_odd, 0, nullptr, 0, 0,
                          0);
      else {
        // a warp without a unit in this tile computes on stale rows (its
        // result is never stored): only live rows count for the range check
        uint32_t tile_bad = 0;
        poly_stage_small<kIn>(mine, minep, ldt_off,
                              slotp + C::kRowsBytes + warp * 8 * C::kPackBytes, ab, cb_lo, cb_hi,
                              w_even, w_odd, lane, &tile_bad);
        if (u_begin + k * W + warp < u_end) bad |= tile_bad;
      }
      cta_sync_named();
      block_stage<false, W>(slot, slotp, blk0, ldc_off, stc_off, ac, cc);
      fence_proxy_async_smem();
      cta_sync_named();
      issue_store(k, slot_i);
    } else {
      block_stage<true, W>(slot, slotp, blk0, ldc_off, stc_off, ac, cc);
      cta_sync_named();
      const int unit = u_begin + k * W + warp;
      const int sg = kAdd ? seg_of(unit) : 0;
      poly_stage<true, kAdd>(mine, minep, ldt_off, am, cm_lo, cm_hi, cb, 0, 0, w_nat,
                             kAdd ? seg_addend(sg) : nullptr,
                             8 * (unit - seg_first(sg)), kAdd ? seg_npoly(sg) : 0,
                             8u * g8 + q4);
      fence_proxy_async_smem();
      __syncwarp();
      issue_store(k, slot_i);
    }
    if (++slot_i == C::kSlots) {
      slot_i = 0;
      phase ^= 1u;
    }
  }
  if (lane == 0) bulk_wait_all();
  if (kIn == kInSmall && __any_sync(0xffffffffu, bad != 0) && lane == 0) atomicOr(&g_status, 4u);
}

// -------------------------------------------------- matrix-vector tiles ---
// k_matvec_tiles: ML-KEM matrix-vector jobs of up to kMaxSegs batches (one k
// each) in one launch,
//     out_i = invntt( sum_j basemul(A_ij, ntt(s_j)) ) + e_i,
// with all three steps on one CTA's shared memory.  A tile is kJobs(k)
// consecutive jobs of one batch, i.e. kRows(k) = kJobs * k consecutive vector
// rows of its s / e / out (32 for k = 2, 4; 24 for k = 3): 8-row TMA boxes in,
// the forward NTT in place (the batch kernels' stages: by polynomial, CTA
// barrier, by block over the tile's n-tiles), the basemul-accumulate by job
// (warp w: jobs w, w+4, ...; ntt(s) from shared memory, all k^2 loads of A from
// global memory issued first, A and e prefetched into L2 one tile ahead with
// bulk prefetches), the inverse NTT plus e in place on the accumulator tile (e
// read in stage B, as the batch inverse with addend), 8-row TMA boxes out.
// Tiles are numbered across the batches (batch b owns [first_tile[b],
// first_tile[b+1])) and CTA c takes tiles c, c + G, c + 2G, ... (G CTAs), so
// the launch has one tail for all batches and its CTAs run one k at a time.  s tiles are double-buffered (the next
// tile's load runs under this tile's work); the accumulator tile is reused
// once its previous store has been read out.  Rows past a batch are out of
// bounds of its tensor maps (zero-filled in; boxes that start past it are
// neither loaded nor stored) and jobs past it are skipped.  The stage
// constants are re-read from L1 at each stage, so that between stages their
// registers hold the basemul's loads in flight.  Every mbarrier wait is
// bounded (2 s; sets status bit 4 and stops the CTA).
struct MvTiles {
  CUtensorMap s_map[kMaxSegs];    // s rows [njobs * k][128 words], 8 x 132-word boxes
  CUtensorMap out_map[kMaxSegs];  // out rows, the same shape (may equal s_map: in place)
  const int16_t* A[kMaxSegs];     // [njobs][k][k][256]
  const uint32_t* e[kMaxSegs];    // [njobs][k][256] as words, or null
  int njobs[kMaxSegs];
  int k[kMaxSegs];
  int first_tile[kMaxSegs + 1];
  int nb;
};

__device__ int32_t g_tile_z[128];  // basemul pair roots z_t (build_pair_roots)
// The tiled kernel's inverse: g_inv with stage B scaled by 2^-16, the factor
// its basemul leaves out (basemul_row_z).
__device__ InvFrags g_tile_inv;

constexpr int kTileSlotBytes = 32 * kRowBytes;      // one 32-row slot
constexpr int kTileSmem = 3 * kTileSlotBytes + 16;  // s slot x 2, accumulators, 2 mbarriers
__host__ __device__ constexpr int tile_units(int k) { return k == 3 ? 3 : 4; }
__host__ __device__ constexpr int tile_jobs(int k) { return 8 * tile_units(k) / k; }

__global__ void __launch_bounds__(128, 4) k_matvec_tiles(const __grid_constant__ MvTiles P) {
  constexpr int W = 4, PP = 2;  // PP: block pairs per warp
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int ntiles = P.first_tile[P.nb];
  // tiles c, c + G, c + 2G, ...: all CTAs move through the batches together
  // (one k's code at a time)
  const int G = (int)gridDim.x;
  const int nmine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / G + 1 : 0;
  const uint32_t smem0 = smem_u32(smem);
  const uint32_t acc = smem0 + 2 * kTileSlotBytes;
  uint8_t* const accp = smem + 2 * kTileSlotBytes;
  const uint32_t bar0 = smem0 + 3 * kTileSlotBytes;

  const int blk0 = 4 * warp;
  int32_t zc[PP][2][2];
#pragma unroll
  for (int p = 0; p < PP; p++)
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int s = 0; s < 2; s++) zc[p][h][s] = 0;
  auto load_am = [&](const uint32_t (*src)[32][4], uint32_t (&am)[2][4]) {
#pragma unroll
    for (int g = 0; g < 2; g++) {
      const uint4 v = ldg_keep_u4(&src[g][lane][0]);
      am[g][0] = v.x;
      am[g][1] = v.y;
      am[g][2] = v.z;
      am[g][3] = v.w;
    }
  };
  auto load_ac = [&](const uint32_t (*src)[2][32][2], uint32_t (&ac)[PP][2][2][2]) {
#pragma unroll
    for (int p = 0; p < PP; p++)
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int s = 0; s < 2; s++) {
          const uint2 v = ldg_keep_u2(&src[blk0 + 2 * p + h][s][lane][0]);
          ac[p][h][s][0] = v.x;
          ac[p][h][s][1] = v.y;
        }
  };
  uint32_t zt[4];
#pragma unroll
  for (int u = 0; u < 4; u++) zt[u] = (uint32_t)g_tile_z[4 * lane + u];

  if (tid == 0) {
    mbar_init(bar0, W);
    mbar_init(bar0 + 8, W);
    fence_mbar_init();
  }
  __syncthreads();
  grid_dependency_wait();
  grid_launch_dependents();
  if (nmine <= 0) return;

  const int q4 = lane & 3, g8 = lane >> 2;
  const uint32_t ldt_off = 32u * ((lane & 7) + 8 * ((lane >> 3) & 1)) + 16u * (lane >> 4);
  const uint32_t hb1 = (lane >> 4) & 1;
  const uint32_t w_even = 32u * g8 + 16u * hb1 + 4u * q4;
  const uint32_t w_odd = 32u * g8 + 16u * (hb1 ^ 1) + 4u * q4;
  const uint32_t w_nat = 32u * g8 + 4u * q4;
  const uint32_t hbw = (uint32_t)((blk0 >> 2) & 1);
  const uint32_t ldc_base = kRowBytes * (lane & 7) + 32u * (lane >> 4);
  const uint32_t ldc_fwd = ldc_base + 16u * (((lane >> 3) & 1) ^ hbw);
  const uint32_t ldc_inv = ldc_base + 16u * ((lane >> 3) & 1);
  const uint32_t stc_off = kRowBytes * (2 * q4) + 4u * g8;
  // the inverse's intermediate with block halves swapped where bit 2 of the
  // block is set (as the batch kernel's): stage A's stores, stage B's rows
  const uint32_t stc_inv = kRowBytes * (2 * q4) + 4u * (g8 ^ (4 * hbw));
  const uint32_t ldt_inv = 32u * ((lane & 7) + 8 * ((lane >> 3) & 1)) +
                           16u * ((lane >> 4) ^ ((lane >> 2) & 1));

  auto batch_of = [&](int t) {
    int b = 0;
#pragma unroll
    for (int j = 1; j < kMaxSegs; j++) b += (j < P.nb && t >= P.first_tile[j]);
    return b;
  };
  auto issue_load = [&](int k, int slot_i) {
    if (lane != 0) return;
    const uint32_t bar = bar0 + 8 * slot_i;
    const int t = (int)blockIdx.x + k * G, b = batch_of(t), kb = P.k[b];
    const int row = (t - P.first_tile[b]) * 8 * tile_units(kb) + 8 * warp;
    if (warp < tile_units(kb) && row < P.njobs[b] * kb) {  // boxes past the batch: none
      mbar_expect_tx(bar, kWarpBoxBytes);
      tma_load_2d(smem0 + slot_i * kTileSlotBytes + warp * kWarpBoxBytes, &P.s_map[b], 0, row,
                  bar);
    } else {
      mbar_expect_tx(bar, 0);  // arrive only
    }
  };
  // A and e of tile k into L2 (one thread; the ranges stop at the batch end),
  // issued as tile k starts: they arrive during its forward NTT.  One tile
  // ahead measured 11 % slower, two tiles ahead slower still (likely the
  // prefetched tiles of all CTAs competing for L2 while they wait there).
  auto prefetch = [&](int k) {
    if (tid != 0) return;
    const int t = (int)blockIdx.x + k * G, b = batch_of(t), kb = P.k[b];
    const int j0 = (t - P.first_tile[b]) * tile_jobs(kb);
    const int nj = min(tile_jobs(kb), P.njobs[b] - j0);
    bulk_prefetch_l2(P.A[b] + (size_t)j0 * kb * kb * 256, (uint32_t)nj * kb * kb * 512u);
    if (P.e[b]) bulk_prefetch_l2(P.e[b] + (size_t)j0 * kb * 128, (uint32_t)nj * kb * 512u);
  };

  // A tile's three phases.  The NTT phases depend on the tile's unit count
  // only (4 for k = 2, 4; 3 for k = 3), so k = 2 and k = 4 share their code.
  // forward NTT of the s tile (in the given slot), in place
  auto fwd_phase = [&](auto nc, uint32_t slot, uint8_t* slotp) {
    constexpr int NU = decltype(nc)::value;
    if (warp < NU) {
      uint32_t fam[2][4];
      load_am(g_fwd.s1, fam);
      const uint2 c1 = ldg_keep_u2(&g_fwd.c1[lane][0]);
      const int32_t cbz[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
      poly_stage<false>(slot + 8 * warp * kRowBytes, slotp + 8 * warp * kRowBytes, ldt_off, fam,
                        (int32_t)c1.x, (int32_t)c1.y, cbz, w_even, w_odd, 0, nullptr, 0, 0, 0);
    }
    cta_sync_named();
    uint32_t fac[PP][2][2][2];
    load_ac(g_fwd.s2, fac);
    block_stage<false, W, PP, NU>(slot, slotp, blk0, ldc_fwd, stc_off, fac, zc);
  };
  // basemul-accumulate into the accumulator tile, one job per warp at a
  // time, all k^2 loads of A issued first
  auto basemul_phase = [&](auto kc, int b, int tl, const uint8_t* slotp) {
    constexpr int K = decltype(kc)::value;
    constexpr int kJobs = tile_jobs(K);
    const int njobs = P.njobs[b];
    for (int jl = warp; jl < kJobs; jl += W) {
      const int job = tl * kJobs + jl;
      if (job >= njobs) break;  // warp-uniform
      const int16_t* Aj = P.A[b] + (size_t)job * K * K * 256 + 8 * lane;
      uint4 a[K][K], bv[K];
      uint2 zb[K];
#pragma unroll
      for (int i = 0; i < K; i++)
#pragma unroll
        for (int j = 0; j < K; j++) a[i][j] = __ldcs((const uint4*)(Aj + (i * K + j) * 256));
#pragma unroll
      for (int j = 0; j < K; j++) {
        bv[j] = *(const uint4*)(slotp + (jl * K + j) * kRowBytes + 16 * lane);
        zb[j] = pair_zb(bv[j], zt);
      }
#pragma unroll
      for (int i = 0; i < K; i++)
        *(uint4*)(accp + (jl * K + i) * kRowBytes + 16 * lane) = basemul_row_z<K>(a[i], bv, zb);
    }
  };
  // inverse NTT plus e on the accumulator tile, in place; then the store
  auto inv_phase = [&](auto nc, int b, int row0, int nvec) {
    constexpr int NU = decltype(nc)::value;
    {
      uint32_t iac[PP][2][2][2];
      load_ac(g_inv.sa, iac);
      block_stage<true, W, PP, NU>(acc, accp, blk0, ldc_inv, stc_inv, iac, zc);
    }
    cta_sync_named();
    if (warp < NU) {
      uint32_t iam[2][4];
      load_am(g_tile_inv.sb, iam);
      int32_t cb[2][4];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const uint4 v = ldg_keep_u4(&g_tile_inv.cbz[lane][t][0]);
        cb[t][0] = (int32_t)v.x;
        cb[t][1] = (int32_t)v.y;
        cb[t][2] = (int32_t)v.z;
        cb[t][3] = (int32_t)v.w;
      }
      poly_stage<true, true>(acc + 8 * warp * kRowBytes, accp + 8 * warp * kRowBytes, ldt_inv, iam,
                             0, 0, cb, 0, 0, w_nat, P.e[b], row0 + 8 * warp, nvec, 8u * g8 + q4);
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0 && row0 + 8 * warp < nvec)  // boxes past the batch are dropped
        tma_store_2d(&P.out_map[b], 0, row0 + 8 * warp, acc + warp * kWarpBoxBytes);
    }
    if (lane == 0) bulk_commit();  // every lane-0 keeps one (possibly empty) group per tile
  };
  using U3 = std::integral_constant<int, 3>;
  using U4 = std::integral_constant<int, 4>;

  issue_load(0, 0);
  for (int k = 0; k < nmine; k++) {
    const int slot_i = k & 1;
    const uint32_t slot = smem0 + slot_i * kTileSlotBytes;
    uint8_t* const slotp = smem + slot_i * kTileSlotBytes;
    const bool ok = mbar_wait_bounded(bar0 + 8 * slot_i, (uint32_t)(k >> 1) & 1u, kWaitLimitNs);
    if (!__syncthreads_and(ok)) {  // CTA-uniform give-up
      if (tid == 0) atomicOr(&g_status, 16u);
      break;
    }
    prefetch(k);
    // the other slot held tile k-1's s, finished before the barrier above
    if (k + 1 < nmine) issue_load(k + 1, slot_i ^ 1);
    const int t = (int)blockIdx.x + k * G, b = batch_of(t), tl = t - P.first_tile[b];
    const int kb = P.k[b];  // CTA-uniform
    const int row0 = tl * 8 * tile_units(kb), nvec = P.njobs[b] * kb;
    if (tile_units(kb) == 3)  // the phase code for the tile's unit count
      fwd_phase(U3{}, slot, slotp);
    else
      fwd_phase(U4{}, slot, slotp);
    if (lane == 0) bulk_wait_read<0>();  // the accumulators' last store has been read out
    cta_sync_named();
    switch (kb) {
      case 2: basemul_phase(std::integral_constant<int, 2>{}, b, tl, slotp); break;
      case 3: basemul_phase(std::integral_constant<int, 3>{}, b, tl, slotp); break;
      default: basemul_phase(std::integral_constant<int, 4>{}, b, tl, slotp); break;
    }
    cta_sync_named();
    if (tile_units(kb) == 3)  // the phase code for the tile's unit count
      inv_phase(U3{}, b, row0, nvec);
    else
      inv_phase(U4{}, b, row0, nvec);
  }
  if (lane == 0) bulk_wait_all();
}

// ------------------------------------------------------------ host side ----
struct Variant {
  const void* fn;
  int threads;
  int smem;
  int tile;
};

template <bool I, int W, int S, int kIn = kInInt16, bool kAdd = false, class P = OneSeg,
          bool kWide = false>
constexpr Variant make_variant() {
  using C = Cfg<W, S, kIn, kWide>;
  return Variant{(const void*)k_ntt_mma<I, W, S, kIn, kAdd, P, kWide>, C::kThreads, C::kSmem,
                 C::kTile};
}

// [inverse][variant] (the mma.sync variants; variant 4 is tk_tc5.cu's)
static const Variant kVariants[2][kNumMmaSyncVariants] = {
    {make_variant<false, 4, 3>(), make_variant<false, 8, 3>(), make_variant<false, 4, 2>(),
     make_variant<false, 4, 2, kInInt16, false, OneSeg, true>()},
    {make_variant<true, 4, 3>(), make_variant<true, 8, 3>(), make_variant<true, 4, 2>(),
     make_variant<true, 4, 2, kInInt16, false, OneSeg, true>()},
};
// Inverse with an addend (the matrix-vector pipeline's iNTT + e), per variant;
// the plain inverse does not carry the addend's loads and adds.
static const Variant kAddVariants[kNumMmaSyncVariants] = {
    make_variant<true, 4, 3, kInInt16, true>(), make_variant<true, 8, 3, kInInt16, true>(),
    make_variant<true, 4, 2, kInInt16, true>(),
    make_variant<true, 4, 2, kInInt16, true, OneSeg, true>()};
// Launches over several segments (the default variants' shapes: forward 3,
// inverse 0): forward, inverse, inverse with addend.  Kept apart so that
// single-batch launches carry none of the segment lookup.
static const Variant kMultiVariants[3] = {
    make_variant<false, 4, 2, kInInt16, false, SegMaps, true>(),
    make_variant<true, 4, 3, kInInt16, false, SegMaps>(),
    make_variant<true, 4, 3, kInInt16, true, SegMaps>()};

// Forward kernels for the small / packed input forms: variant 3's shape (4
// warps, 2 slots, stage-1 sums kept as int32 in shared memory; 3 CTAs/SM).
static const Variant kFormVariants[kNumInputForms] = {
    make_variant<false, 4, 2, kInSmall, false, OneSeg, true>(),
    make_variant<false, 4, 2, kInPack2, false, OneSeg, true>(),
    make_variant<false, 4, 2, kInPack3, false, OneSeg, true>()};

static thread_local int g_last_encode_result = 0;

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// The batch as a [npoly][128] uint32 tensor; boxes of 8 polynomials x 132
// words (the last 4 words are out of bounds: the smem row pad).
static bool encode_batch_map(CUtensorMap* map, const int16_t* base, int npoly) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) {
    g_last_encode_result = -1;
    return false;
  }
  const cuuint64_t dims[2] = {128, (cuuint64_t)npoly};
  const cuuint64_t strides[1] = {512};
  const cuuint32_t box[2] = {kRowBytes / 4, 8};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r =
      enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, (void*)base, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  g_last_encode_result = (int)r;
  return r == CUDA_SUCCESS;
}

// A packed batch as a [npoly][row_bytes / 4] uint32 tensor, boxes of 8 rows.
static bool encode_packed_map(CUtensorMap* map, const void* base, int npoly, int row_bytes) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) {
    g_last_encode_result = -1;
    return false;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)(row_bytes / 4), (cuuint64_t)npoly};
  const cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)(row_bytes / 4), 8};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r =
      enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, (void*)base, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  g_last_encode_result = (int)r;
  return r == CUDA_SUCCESS;
}

int last_encode_result() { return g_last_encode_result; }
void note_encode_result(int r) { g_last_encode_result = r; }

static bool upload_tables_current_device() {
  static Matrices M, MR;
  static FwdFrags FF;
  static InvFrags IF, IFR;
  static std::once_flag once;
  std::call_once(once, [] {
    build_matrices(&M);
    build_fwd_frags(M, &FF);
    build_inv_frags(M, &IF);
    MR = M;
    scale_inverse(&MR, kRinv);
    build_inv_frags(MR, &IFR);
  });
  if (cudaMemcpyToSymbol(g_fwd, &FF, sizeof(FF)) != cudaSuccess) return false;
  if (cudaMemcpyToSymbol(g_inv, &IF, sizeof(IF)) != cudaSuccess) return false;
  if (cudaMemcpyToSymbol(g_tile_inv, &IFR, sizeof(IFR)) != cudaSuccess) return false;
  int32_t z[128];
  build_pair_roots(z);
  if (cudaMemcpyToSymbol(g_tile_z, z, sizeof(z)) != cudaSuccess) return false;
  const unsigned zero = 0;
  return cudaMemcpyToSymbol(g_status, &zero, sizeof(zero)) == cudaSuccess;
}

bool mma_init_device(DeviceInfo* info) {
  if (!upload_tables_current_device()) return false;
  void* st = nullptr;
  if (cudaGetSymbolAddress(&st, g_status) != cudaSuccess || !st) return false;
  info->status = (unsigned*)st;
  for (int inv = 0; inv < 2; inv++)
    for (int v = 0; v < kNumMmaSyncVariants; v++) {
      const Variant& V = kVariants[inv][v];
      if (cudaFuncSetAttribute(V.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, V.smem) !=
          cudaSuccess)
        return false;
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, V.fn, V.threads, V.smem) !=
          cudaSuccess)
        return false;
      info->mma_ctas_per_sm[inv][v] = per_sm > 0 ? per_sm : 1;
    }
  for (int v = 0; v < kNumMmaSyncVariants; v++) {
    const Variant& V = kAddVariants[v];
    if (cudaFuncSetAttribute(V.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, V.smem) !=
        cudaSuccess)
      return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, V.fn, V.threads, V.smem) !=
        cudaSuccess)
      return false;
    info->add_ctas_per_sm[v] = per_sm > 0 ? per_sm : 1;
  }
  for (int m = 0; m < 3; m++) {
    const Variant& V = kMultiVariants[m];
    if (cudaFuncSetAttribute(V.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, V.smem) !=
        cudaSuccess)
      return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, V.fn, V.threads, V.smem) !=
        cudaSuccess)
      return false;
    info->multi_ctas_per_sm[m] = per_sm > 0 ? per_sm : 1;
  }
  {
    const void* fn = (const void*)k_matvec_tiles;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem) !=
        cudaSuccess)
      return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, kTileSmem) != cudaSuccess)
      return false;
    info->tile_ctas_per_sm = per_sm > 0 ? per_sm : 1;
  }
  for (int f = 0; f < kNumInputForms; f++) {
    const Variant& V = kFormVariants[f];
    if (cudaFuncSetAttribute(V.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, V.smem) !=
        cudaSuccess)
      return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, V.fn, V.threads, V.smem) !=
        cudaSuccess)
      return false;
    info->form_ctas_per_sm[f] = per_sm > 0 ? per_sm : 1;
  }
  return true;
}

template <class P>
static cudaError_t launch_variant(const Variant& V, long long cap, const P& m, long long polys,
                                  cudaStream_t stream) {
  long long ctas = (polys + V.tile - 1) / V.tile;
  if (ctas > cap) ctas = cap;
  if (ctas < 1) ctas = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ctas);
  cfg.blockDim = dim3((unsigned)V.threads);
  cfg.dynamicSmemBytes = (size_t)V.smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[1] = {(void*)&m};
  return cudaLaunchKernelExC(&cfg, V.fn, args);
}

cudaError_t launch_fwd_form(int form, const void* src, int16_t* dst, long long npoly,
                            const DeviceInfo& info, cudaStream_t stream) {
  if (form < 1 || form > kNumInputForms) return cudaErrorInvalidValue;
  const Variant& V = kFormVariants[form - 1];
  const long long cap = (long long)info.num_sms * info.form_ctas_per_sm[form - 1];
  const int row_bytes = form == kInPack2 ? 64 : form == kInPack3 ? 128 : 512;
  for (long long done = 0; done < npoly; done += kMaxLaunchPolys) {
    const int n = (int)((npoly - done) < kMaxLaunchPolys ? (npoly - done) : kMaxLaunchPolys);
    const uint8_t* in = (const uint8_t*)src + done * row_bytes;
    OneSeg m = {};
    const bool ok_in = form == kInSmall ? encode_batch_map(&m.in, (const int16_t*)in, n)
                                        : encode_packed_map(&m.in, in, n, row_bytes);
    if (!ok_in) return cudaErrorInvalidResourceHandle;
    if ((const void*)in == (const void*)(dst + done * 256))
      m.out = m.in;
    else if (!encode_batch_map(&m.out, dst + done * 256, n))
      return cudaErrorInvalidResourceHandle;
    m.npoly = n;
    const cudaError_t e = launch_variant(V, cap, m, n, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// One piece (at most kMaxLaunchPolys polynomials: TMA coordinates are 32-bit).
struct Piece {
  const int16_t* src;
  int16_t* dst;
  int n;
  const int16_t* addend;
};

cudaError_t launch_mma_segs(bool inverse, int variant, const Seg* segs, int nseg,
                            const DeviceInfo& info, cudaStream_t stream) {
  if (!variant_valid(inverse, variant)) variant = 0;
  bool add_form = false;
  for (int j = 0; j < nseg; j++) add_form |= inverse && segs[j].addend != nullptr;
  // the tcgen05 kernels: plain batches, one launch each; the inverse with an
  // addend runs the mma.sync shapes
  if (variant == kTc5Variant) {
    if (!add_form) {
      for (int j = 0; j < nseg; j++) {
        const cudaError_t e = launch_tc5(inverse, segs[j].src, segs[j].dst, segs[j].npoly, info,
                                         stream);
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    }
    variant = 0;
  }
  // pieces of at most kMaxLaunchPolys, in order
  Piece pc[kMaxSegs] = {};
  int np = 0;
  auto launch_pieces = [&]() -> cudaError_t {
    if (np == 0) return cudaSuccess;
    if (np == 1) {  // one batch: the compact single-segment kernels
      const Variant& V = add_form ? kAddVariants[variant] : kVariants[inverse ? 1 : 0][variant];
      const long long cap = (long long)info.num_sms *
                            (add_form ? info.add_ctas_per_sm[variant]
                                      : info.mma_ctas_per_sm[inverse ? 1 : 0][variant]);
      OneSeg m = {};
      if (!encode_batch_map(&m.in, pc[0].src, pc[0].n)) return cudaErrorInvalidResourceHandle;
      if (pc[0].src == pc[0].dst)
        m.out = m.in;
      else if (!encode_batch_map(&m.out, pc[0].dst, pc[0].n))
        return cudaErrorInvalidResourceHandle;
      m.addend = (const uint32_t*)pc[0].addend;
      m.npoly = pc[0].n;
      np = 0;
      return launch_variant(V, cap, m, m.npoly, stream);
    }
    const int which = !inverse ? 0 : add_form ? 2 : 1;
    const Variant& V = kMultiVariants[which];
    const long long cap = (long long)info.num_sms * info.multi_ctas_per_sm[which];
    SegMaps m = {};
    int units = 0;
    for (int k = 0; k < np; k++) {
      if (!encode_batch_map(&m.in[k], pc[k].src, pc[k].n)) return cudaErrorInvalidResourceHandle;
      if (pc[k].src == pc[k].dst)
        m.out[k] = m.in[k];
      else if (!encode_batch_map(&m.out[k], pc[k].dst, pc[k].n))
        return cudaErrorInvalidResourceHandle;
      m.addend[k] = (const uint32_t*)pc[k].addend;
      m.npoly[k] = pc[k].n;
      m.first_unit[k] = units;
      units += (pc[k].n + 7) / 8;
    }
    m.first_unit[np] = units;
    m.nseg = np;
    np = 0;
    return launch_variant(V, cap, m, 8LL * units, stream);
  };
  for (int j = 0; j < nseg; j++) {
    const Seg& g = segs[j];
    for (long long done = 0; done < g.npoly; done += kMaxLaunchPolys) {
      const int n = (int)((g.npoly - done) < kMaxLaunchPolys ? (g.npoly - done) : kMaxLaunchPolys);
      pc[np++] = Piece{g.src + done * 256, g.dst + done * 256, n,
                       g.addend ? g.addend + done * 256 : nullptr};
      if (np == kMaxSegs) {
        const cudaError_t e = launch_pieces();
        if (e != cudaSuccess) return e;
      }
    }
  }
  return launch_pieces();
}

cudaError_t launch_mma(bool inverse, int variant, const int16_t* src, int16_t* dst,
                       long long npoly, const DeviceInfo& info, cudaStream_t stream,
                       const int16_t* addend) {
  const Seg g{src, dst, npoly, addend};
  return launch_mma_segs(inverse, variant, &g, 1, info, stream);
}

cudaError_t launch_matvec_tile(const MatvecPart* batches, int nb, const DeviceInfo& info,
                               cudaStream_t stream) {
  if (nb > kMaxSegs) return cudaErrorInvalidValue;
  MvTiles m = {};
  for (int b = 0; b < nb; b++) {
    const MatvecPart& B = batches[b];
    // rows are 32-bit TMA coordinates and tile numbers 32-bit integers
    if (B.njobs * (size_t)B.k > (size_t)kMaxLaunchPolys) return cudaErrorInvalidValue;
    const int nvec = (int)(B.njobs * B.k);
    if (!encode_batch_map(&m.s_map[b], B.s, nvec)) return cudaErrorInvalidResourceHandle;
    if (B.out == B.s)
      m.out_map[b] = m.s_map[b];
    else if (!encode_batch_map(&m.out_map[b], B.out, nvec))
      return cudaErrorInvalidResourceHandle;
    m.A[b] = B.A;
    m.e[b] = (const uint32_t*)B.e;
    m.njobs[b] = (int)B.njobs;
    m.k[b] = B.k;
    const int tj = tile_jobs(B.k);
    m.first_tile[b + 1] = m.first_tile[b] + (int)((B.njobs + tj - 1) / tj);
  }
  m.nb = nb;
  long long ctas = m.first_tile[nb];
  if (ctas <= 0) return cudaSuccess;
  const long long cap = (long long)info.num_sms * info.tile_ctas_per_sm;
  if (ctas > cap) ctas = cap;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ctas);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = (size_t)kTileSmem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* args[1] = {(void*)&m};
  return cudaLaunchKernelExC(&cfg, (const void*)k_matvec_tiles, args);
}

// Self-test of the give-up path: one CTA waits, through the same bounded
// wait as the batch kernels, on an mbarrier that no thread arrives at; after
// limit_ns it sets status bit 3 and returns (the wait ends by design).
__global__ void k_selftest_wait(unsigned long long limit_ns) {
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t b = smem_u32(&bar);
  if (threadIdx.x == 0) {
    mbar_init(b, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(b, 0, limit_ns);
  if (!__syncthreads_and(ok) && threadIdx.x == 0) atomicOr(&g_status, 8u);
}

cudaError_t launch_selftest_wait(unsigned long long limit_ns, cudaStream_t stream) {
  k_selftest_wait<<<1, 32, 0, stream>>>(limit_ns);
  return cudaGetLastError();
}

cudaError_t read_and_clear_status(unsigned* flags) {
  unsigned v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_status, sizeof(v));
  if (e != cudaSuccess) return e;
  if (v) {
    const unsigned zero = 0;
    e = cudaMemcpyToSymbol(g_status, &zero, sizeof(zero));
  }
  *flags = v;
  return e;
}

}  // namespace tk
