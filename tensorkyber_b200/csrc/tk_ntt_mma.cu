// tk_ntt_mma.cu -- batched ML-KEM NTT / iNTT on sm_100a: TMA bulk staging +
// int8 mma.sync tiles, one independent pipeline per warp.
//
// Work unit: 8 consecutive polynomials (4 KiB).  Each warp owns kSlots smem
// slots of 8 padded rows (528 B per polynomial, the 16 B pad makes every
// access pattern below bank-conflict free or 2-way at most) and streams units
// u = warp_id, warp_id + n_warps, ... through them:
//
//   TMA  cp.async.bulk global->smem, 8 x 512 B, completion on an mbarrier
//   fwd  stage 1 (M1, per polynomial): ldmatrix.trans -> 4 x m16n8k32 s8.u8
//        -> S = D_lo + 128 D_hi -> lazy Barrett -> parity-split rows in place
//        stage 2 (M2, per block pair, 8 polynomials): ldmatrix -> 4 x
//        m16n8k16 -> exact Barrett to [0, q) -> natural order in place
//   inv  stage A (MA, per block): 8 B loads + byte_perm -> 2 x m16n8k16
//        -> lazy Barrett -> natural order in place
//        stage B (Minv, per polynomial): like fwd stage 1, output centred
//   TMA  cp.async.bulk smem->global, 8 x 512 B; the slot is refilled once
//        the store has been read out (wait_group.read).
//
// Reference counterparts: k_ntt_2tc_tc_cc / k_invntt_2tc_tc_cc and
// k_ntt_tc_cc_cp / k_invntt_tc_cc_cp (ntt_bench/ntt_bench.cu:61-131,
// 181-277) with ntt_core / intt_core (ntt_bench/ntt_kernels.cuh:393-489,
// 548-625).
#include <cuda_runtime.h>
#include <stdint.h>

#include "tk_internal.h"
#include "tk_ptx.cuh"
#include "tk_tables.h"

namespace tk {

constexpr int kRowBytes = 528;                  // 512 B polynomial + 16 B pad
constexpr int kUnit = 8;                        // polynomials per warp unit
constexpr int kSlotBytes = kUnit * kRowBytes;   // 4224
constexpr int kSlots = 3;                       // pipeline depth per warp
constexpr int kWarpSmem = kSlots * kSlotBytes + 64;  // + mbarriers
constexpr int kWarpsPerCta = 4;
constexpr int kCtaThreads = 32 * kWarpsPerCta;
constexpr int kCtaSmem = kWarpsPerCta * kWarpSmem;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s bound on every mbarrier wait

__device__ FwdFrags g_fwd;
__device__ InvFrags g_inv;
__device__ unsigned int g_status;

// ---------------------------------------------------------------- forward --
struct FwdRegs {
  uint32_t a1[2][4];
  int32_t c1lo, c1hi;
  uint32_t a2[16][2][2];
};

__device__ __forceinline__ void load_fwd_regs(FwdRegs& R, int lane) {
#pragma unroll
  for (int g = 0; g < 2; g++)
#pragma unroll
    for (int j = 0; j < 4; j++) R.a1[g][j] = g_fwd.s1[g][lane][j];
  R.c1lo = g_fwd.c1[lane][0];
  R.c1hi = g_fwd.c1[lane][1];
#pragma unroll
  for (int b = 0; b < 16; b++)
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
      for (int j = 0; j < 2; j++) R.a2[b][s][j] = g_fwd.s2[b][s][lane][j];
}

// Stage 1 of one polynomial whose row starts at smem address rb.
__device__ __forceinline__ void fwd_stage1(const FwdRegs& R, uint32_t rb, uint32_t ld_off,
                                           uint8_t* row, uint32_t w_even, uint32_t w_odd) {
  uint32_t b0, b1, b2, b3;
  ldsm_x4_t(rb + ld_off, b0, b1, b2, b3);
  // x ^ 0x8000 = x + 32768 as an unsigned 16-bit value; the 32768 * rowsum
  // term is cancelled by the group-0 accumulator init (c1).
  b0 ^= 0x80008000u;
  b1 ^= 0x80008000u;
  b2 ^= 0x80008000u;
  b3 ^= 0x80008000u;
  const int32_t cinit[4] = {R.c1lo, R.c1lo, R.c1hi, R.c1hi};
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k32(lo0, R.a1[0], b0, b1, cinit);
  mma_k32(hi0, R.a1[1], b0, b1, zero);
  mma_k32(lo1, R.a1[0], b2, b3, cinit);
  mma_k32(hi1, R.a1[1], b2, b3, zero);
  uint32_t y0[4], y1[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    y0[e] = red_lazy((uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7));
    y1[e] = red_lazy((uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7));
  }
  // regs: [0] (row i, c=2q), [1] (row i, c=2q+1), [2] (row i+8, c=2q), [3] (row i+8, c=2q+1);
  // n-tile 1 is c+8.  Parity-split slots: (c=2q | c=8+2q) and (c=2q+1 | c=9+2q).
  *(uint32_t*)(row + w_even) = pack2(y0[0], y1[0]);
  *(uint32_t*)(row + w_odd) = pack2(y0[1], y1[1]);
  *(uint32_t*)(row + w_even + 256) = pack2(y0[2], y1[2]);
  *(uint32_t*)(row + w_odd + 256) = pack2(y0[3], y1[3]);
}

template <int I>
__device__ __forceinline__ void fwd_stage2_pair(const FwdRegs& R, uint32_t slot, uint8_t* slotp,
                                                uint32_t ld_off_h0, uint32_t ld_off_h1,
                                                uint32_t st_off) {
  uint32_t r[4];
  constexpr int hb = (I >> 2) & 1;
  ldsm_x4(slot + 32 * I + (hb ? ld_off_h1 : ld_off_h0), r[0], r[1], r[2], r[3]);
  const int32_t zero[4] = {0, 0, 0, 0};
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int32_t de[4], dodd[4];
    mma_k16(de, R.a2[I + h][0], r[2 * h], zero);
    mma_k16(dodd, R.a2[I + h][1], r[2 * h + 1], zero);
    const uint32_t e0 = red_exact((uint32_t)de[0] + ((uint32_t)de[2] << 7));
    const uint32_t e1 = red_exact((uint32_t)de[1] + ((uint32_t)de[3] << 7));
    const uint32_t o0 = red_exact((uint32_t)dodd[0] + ((uint32_t)dodd[2] << 7));
    const uint32_t o1 = red_exact((uint32_t)dodd[1] + ((uint32_t)dodd[3] << 7));
    *(uint32_t*)(slotp + st_off + 32 * (I + h)) = pack2(e0, o0);
    *(uint32_t*)(slotp + st_off + kRowBytes + 32 * (I + h)) = pack2(e1, o1);
  }
}

// ---------------------------------------------------------------- inverse --
struct InvRegs {
  uint32_t aa[16][2][2];
  uint32_t ab[2][4];
};

__device__ __forceinline__ void load_inv_regs(InvRegs& R, int lane) {
#pragma unroll
  for (int b = 0; b < 16; b++)
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
      for (int j = 0; j < 2; j++) R.aa[b][s][j] = g_inv.sa[b][s][lane][j];
#pragma unroll
  for (int g = 0; g < 2; g++)
#pragma unroll
    for (int j = 0; j < 4; j++) R.ab[g][j] = g_inv.sb[g][lane][j];
}

template <int B>
__device__ __forceinline__ void inv_stageA_block(const InvRegs& R, uint8_t* slotp,
                                                 uint32_t ld_off, uint32_t st_off) {
  const uint2 v = *(const uint2*)(slotp + ld_off + 32 * B);
  // +10q bias: (x ^ 0x8000) + 522 per 16-bit half, no carry for x <= 32245.
  const uint32_t a = (v.x ^ 0x80008000u) + kBias10qPacked;
  const uint32_t b = (v.y ^ 0x80008000u) + kBias10qPacked;
  const uint32_t ev = __byte_perm(a, b, 0x5410);  // c = 4q, 4q+2
  const uint32_t od = __byte_perm(a, b, 0x7632);  // c = 4q+1, 4q+3
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t de[4], dodd[4];
  mma_k16(de, R.aa[B][0], ev, zero);
  mma_k16(dodd, R.aa[B][1], od, zero);
  const uint32_t e0 = red_lazy((uint32_t)de[0] + ((uint32_t)de[2] << 7));
  const uint32_t e1 = red_lazy((uint32_t)de[1] + ((uint32_t)de[3] << 7));
  const uint32_t o0 = red_lazy((uint32_t)dodd[0] + ((uint32_t)dodd[2] << 7));
  const uint32_t o1 = red_lazy((uint32_t)dodd[1] + ((uint32_t)dodd[3] << 7));
  *(uint32_t*)(slotp + st_off + 32 * B) = pack2(e0, o0);
  *(uint32_t*)(slotp + st_off + kRowBytes + 32 * B) = pack2(e1, o1);
}

__device__ __forceinline__ void inv_stageB(const InvRegs& R, uint32_t rb, uint32_t ld_off,
                                           uint8_t* row, uint32_t w_off) {
  uint32_t b0, b1, b2, b3;
  ldsm_x4_t(rb + ld_off, b0, b1, b2, b3);
  // +(q-1)/2 in the accumulator init so that S - q*floor(S/q) - 1664 is the
  // centred representative in [-(q-1)/2, (q-1)/2].
  const int32_t cinit[4] = {1664, 1664, 1664, 1664};
  const int32_t zero[4] = {0, 0, 0, 0};
  int32_t lo0[4], hi0[4], lo1[4], hi1[4];
  mma_k32(lo0, R.ab[0], b0, b1, cinit);
  mma_k32(hi0, R.ab[1], b0, b1, zero);
  mma_k32(lo1, R.ab[0], b2, b3, cinit);
  mma_k32(hi1, R.ab[1], b2, b3, zero);
  uint32_t y0[4], y1[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    y0[e] = red_exact((uint32_t)lo0[e] + ((uint32_t)hi0[e] << 7)) - 1664u;
    y1[e] = red_exact((uint32_t)lo1[e] + ((uint32_t)hi1[e] << 7)) - 1664u;
  }
  *(uint32_t*)(row + w_off) = pack2(y0[0], y0[1]);
  *(uint32_t*)(row + w_off + 16) = pack2(y1[0], y1[1]);
  *(uint32_t*)(row + w_off + 256) = pack2(y0[2], y0[3]);
  *(uint32_t*)(row + w_off + 256 + 16) = pack2(y1[2], y1[3]);
}

// ------------------------------------------------------------ the kernel ---
template <bool kInverse>
__global__ void __launch_bounds__(kCtaThreads)
    k_ntt_mma(const int16_t* __restrict__ src, int16_t* __restrict__ dst, long long npoly) {
  extern __shared__ __align__(128) uint8_t smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const long long nunits = (npoly + kUnit - 1) / kUnit;
  const long long gw = (long long)blockIdx.x * kWarpsPerCta + warp;
  const long long nw = (long long)gridDim.x * kWarpsPerCta;
  if (gw >= nunits) return;
  const long long nmine = (nunits - gw + nw - 1) / nw;

  uint8_t* wsm = smem + warp * kWarpSmem;
  const uint32_t slot0 = smem_u32(wsm);
  const uint32_t bar0 = slot0 + kSlots * kSlotBytes;

  FwdRegs F;
  InvRegs V;
  if (kInverse)
    load_inv_regs(V, lane);
  else
    load_fwd_regs(F, lane);

  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < kSlots; s++) mbar_init(bar0 + 8 * s, 1);
    fence_mbar_init();
  }
  __syncwarp();

  const int q4 = lane & 3, g8 = lane >> 2;
  // ldmatrix.trans row addresses (stage 1 / stage B): matrix j = lane/8 covers
  // m = (lane&7) + 8*(j&1), coefficients 8*(j>>1) .. +7.
  const uint32_t ldt_off = 32u * ((lane & 7) + 8 * ((lane >> 3) & 1)) + 16u * (lane >> 4);
  // fwd stage-1 stores: row i = lane/4 (and +8), parity halves swapped for
  // blocks with bit 2 set.
  const uint32_t hb = (lane >> 4) & 1;
  const uint32_t w_even = 32u * g8 + 16u * hb + 4u * q4;
  const uint32_t w_odd = 32u * g8 + 16u * (hb ^ 1) + 4u * q4;
  // fwd stage-2 ldmatrix rows: polynomial lane&7, block I + lane/16, half
  // (lane/8)&1 (xor the block's bit 2).
  const uint32_t s2_h0 = kRowBytes * (lane & 7) + 32u * (lane >> 4) + 16u * ((lane >> 3) & 1);
  const uint32_t s2_h1 = kRowBytes * (lane & 7) + 32u * (lane >> 4) + 16u * (((lane >> 3) & 1) ^ 1);
  // outputs of the block-wise stages: polynomial 2*q4 (and +1), pair lane/4.
  const uint32_t st2_off = kRowBytes * (2 * q4) + 4u * g8;
  // inverse stage-A loads: polynomial lane/4, coefficients 4*q4 .. +3.
  const uint32_t la_off = kRowBytes * g8 + 8u * q4;
  // inverse stage-B stores: row i = lane/4, coefficient pair 2*q4.
  const uint32_t wb_off = 32u * g8 + 4u * q4;

  auto issue_load = [&](long long k, int slot_i) {
    const long long u = gw + k * nw;
    const long long left = npoly - u * kUnit;
    const int valid = left < kUnit ? (int)left : kUnit;
    const uint32_t bar = bar0 + 8 * slot_i;
    if (lane == 0) mbar_expect_tx(bar, 512u * valid);
    __syncwarp();
    if (lane < valid)
      bulk_g2s(slot0 + slot_i * kSlotBytes + lane * kRowBytes, src + (u * kUnit + lane) * kN,
               512u, bar);
  };

  issue_load(0, 0);
  if (nmine > 1) issue_load(1, 1);

  int slot_i = 0;
  uint32_t phase = 0;
  for (long long k = 0; k < nmine; k++) {
    const uint32_t slot = slot0 + slot_i * kSlotBytes;
    uint8_t* slotp = wsm + slot_i * kSlotBytes;
    const bool ok = mbar_wait_bounded(bar0 + 8 * slot_i, phase, kWaitLimitNs);
    if (!__all_sync(0xffffffffu, ok)) {  // warp-uniform give-up
      if (lane == 0) atomicOr(&g_status, kInverse ? 2u : 1u);
      break;
    }
    if (!kInverse) {
#pragma unroll 2
      for (int p = 0; p < kUnit; p++)
        fwd_stage1(F, slot + p * kRowBytes, ldt_off, slotp + p * kRowBytes, w_even, w_odd);
      __syncwarp();
      fwd_stage2_pair<0>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<2>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<4>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<6>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<8>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<10>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<12>(F, slot, slotp, s2_h0, s2_h1, st2_off);
      fwd_stage2_pair<14>(F, slot, slotp, s2_h0, s2_h1, st2_off);
    } else {
      inv_stageA_block<0>(V, slotp, la_off, st2_off);
      inv_stageA_block<1>(V, slotp, la_off, st2_off);
      inv_stageA_block<2>(V, slotp, la_off, st2_off);
      inv_stageA_block<3>(V, slotp, la_off, st2_off);
      inv_stageA_block<4>(V, slotp, la_off, st2_off);
      inv_stageA_block<5>(V, slotp, la_off, st2_off);
      inv_stageA_block<6>(V, slotp, la_off, st2_off);
      inv_stageA_block<7>(V, slotp, la_off, st2_off);
      inv_stageA_block<8>(V, slotp, la_off, st2_off);
      inv_stageA_block<9>(V, slotp, la_off, st2_off);
      inv_stageA_block<10>(V, slotp, la_off, st2_off);
      inv_stageA_block<11>(V, slotp, la_off, st2_off);
      inv_stageA_block<12>(V, slotp, la_off, st2_off);
      inv_stageA_block<13>(V, slotp, la_off, st2_off);
      inv_stageA_block<14>(V, slotp, la_off, st2_off);
      inv_stageA_block<15>(V, slotp, la_off, st2_off);
      __syncwarp();
#pragma unroll 2
      for (int p = 0; p < kUnit; p++)
        inv_stageB(V, slot + p * kRowBytes, ldt_off, slotp + p * kRowBytes, wb_off);
    }
    // generic-proxy writes -> async-proxy bulk store
    fence_proxy_async_smem();
    __syncwarp();
    {
      const long long u = gw + k * nw;
      const long long left = npoly - u * kUnit;
      const int valid = left < kUnit ? (int)left : kUnit;
      if (lane < valid) bulk_s2g(dst + (u * kUnit + lane) * kN, slot + lane * kRowBytes, 512u);
      bulk_commit();
    }
    if (k + 2 < nmine) {
      // slot of unit k+2 last held unit k-1: its store must be read out.
      bulk_wait_read<1>();
      int s2 = slot_i + 2;
      if (s2 >= kSlots) s2 -= kSlots;
      issue_load(k + 2, s2);
    }
    if (++slot_i == kSlots) {
      slot_i = 0;
      phase ^= 1u;
    }
  }
  bulk_wait_all();
}

// ------------------------------------------------------------ host side ----
static bool upload_tables_current_device() {
  static Matrices M;
  static FwdFrags FF;
  static InvFrags IF;
  static bool built = false;
  if (!built) {
    build_matrices(&M);
    build_fwd_frags(M, &FF);
    build_inv_frags(M, &IF);
    built = true;
  }
  if (cudaMemcpyToSymbol(g_fwd, &FF, sizeof(FF)) != cudaSuccess) return false;
  if (cudaMemcpyToSymbol(g_inv, &IF, sizeof(IF)) != cudaSuccess) return false;
  const unsigned zero = 0;
  if (cudaMemcpyToSymbol(g_status, &zero, sizeof(zero)) != cudaSuccess) return false;
  if (cudaFuncSetAttribute(k_ntt_mma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kCtaSmem) != cudaSuccess)
    return false;
  if (cudaFuncSetAttribute(k_ntt_mma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kCtaSmem) != cudaSuccess)
    return false;
  return true;
}

bool mma_init_device(DeviceInfo* info) {
  if (!upload_tables_current_device()) return false;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ntt_mma<false>, kCtaThreads,
                                                    kCtaSmem) != cudaSuccess)
    return false;
  int per_sm_inv = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_inv, k_ntt_mma<true>, kCtaThreads,
                                                    kCtaSmem) != cudaSuccess)
    return false;
  info->mma_ctas_per_sm[0] = per_sm > 0 ? per_sm : 1;
  info->mma_ctas_per_sm[1] = per_sm_inv > 0 ? per_sm_inv : 1;
  return true;
}

cudaError_t launch_mma(bool inverse, const int16_t* src, int16_t* dst, long long npoly,
                       const DeviceInfo& info, cudaStream_t stream) {
  const long long nunits = (npoly + kUnit - 1) / kUnit;
  long long ctas = (nunits + kWarpsPerCta - 1) / kWarpsPerCta;
  const long long cap = (long long)info.num_sms * info.mma_ctas_per_sm[inverse ? 1 : 0];
  if (ctas > cap) ctas = cap;
  if (ctas < 1) ctas = 1;
  if (inverse)
    k_ntt_mma<true><<<(unsigned)ctas, kCtaThreads, kCtaSmem, stream>>>(src, dst, npoly);
  else
    k_ntt_mma<false><<<(unsigned)ctas, kCtaThreads, kCtaSmem, stream>>>(src, dst, npoly);
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
