// tk_tc5.cu -- batched ML-KEM NTT and inverse NTT on the 5th-generation
// tensor cores (tcgen05.mma kind::i8, int32 accumulators in tensor memory),
// sm_100a.
//
// Same transforms as the mma.sync kernels (tk_ntt_mma.cu) and the same method
// (TensorKyber's ntt_core / intt_core, ntt_bench/ntt_kernels.cuh:393-489,
// 548-625): forward layers 1-4 as M1 over the block index m, layers 5-7 as the
// per-block M2^(i); inverse stage A as the per-block MA^(m), stage B as Minv
// over m (with the final x1441 Montgomery factor); every constant as two
// 7-bit int8 limbs.  The B200 formulation:
//
//   * A tile is 128 polynomials, the M dimension of every MMA (one polynomial
//     per tensor-memory lane).  TMA loads it as four boxes of 64 coefficients
//     x 128 rows with the 128-byte swizzle, which is exactly the canonical
//     K-major SW128 operand layout: the inverse's stage-A A operand for block
//     m is the 32 bytes of that block in each row, read straight from the
//     loaded tile.  The forward contracts over m first, so the 8 epilogue
//     warps transpose the tile in place into stage 1's operand (K-major
//     without swizzle) before its MMAs.
//   * Signed data need no CUDA-core pass.  An int16 x = b0 + 256 b1 with b0
//     unsigned and b1 signed, so the first stage is two MMAs per block (or
//     coefficient) into the same accumulator: one with unsigned data and
//     constants on the low bytes' K rows, one with signed data and constants
//     256 C mod q on the high bytes' K rows; the other rows of each constant
//     tile are zero.
//   * The first stage's sums S = D_lo + 128 D_hi are never reduced: S + 2048 q
//     (non-negative, below 2^25) goes back to tensor memory as int32,
//     transposed -- output n's second-stage operand is the 16 columns 16 n ..
//     16 n + 15, read by tcgen05.mma straight from tensor memory as 64
//     unsigned bytes whose constants carry 256^j mod q, two MMAs per
//     coefficient (inverse) or block (forward).
//   * The second stage's sums (below 2^26) get one exact reduction (centred
//     for the inverse, [0, q) for the forward), are packed to int16 and
//     written in the TMA layout over the tile's own input slot (its MMAs have
//     finished), and TMA stores the tile.
//
// Roles (320 threads, one CTA per SM by shared memory): warp 9 lane 0 issues
// TMA loads and stores; warp 8 lane 0 issues MMAs (and warp 8 owns the
// tensor-memory allocation); warps 0-7 move data between tensor memory,
// registers and shared memory, warps w and w + 4 sharing tensor-memory lanes
// 32 (w % 4) .. + 31 (polynomials) and splitting the columns.  Tensor memory
// (512 columns): 0-255 the first stage's sums, 256-383 and 384-511 two
// accumulator buffers of four 32-column MMA results each.  Per tile the MMA
// thread issues 8 chunks of four MMA results (8 MMAs each) into the buffers
// in turn; warps 0-3 take buffer 0,
// warps 4-7 buffer 1.  Two input slots of 64 KiB: the load of tile k + 2 goes
// into tile k's slot once tile k's output (written over its input) has been
// read out by the store.  Every mbarrier wait gives up after 2 s (status bit
// 0 forward / 1 inverse, as the other kernels); the MMA thread then drains
// its MMAs and the producer its copies before the CTA frees tensor memory and
// exits.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <mutex>

#include "tk_internal.h"
#include "tk_ptx.cuh"
#include "tk_tables.h"

namespace tk {
namespace {

constexpr int kTcTile = 128;                      // polynomials per tile (MMA M)
constexpr int kTcQuarterBytes = kTcTile * 128;    // one 64-coefficient box: 16 KiB
constexpr int kTcSlotBytes = 4 * kTcQuarterBytes;  // 64 KiB
constexpr int kTcEpiWarps = 8;
constexpr int kTcMmaWarp = 8, kTcTmaWarp = 9;
constexpr int kTcThreads = 32 * (kTcEpiWarps + 2);
// dynamic shared memory, from a 1024-byte aligned base (the swizzle atom):
// two 64 KiB tile slots, this direction's constant tiles, the mbarriers
// (in_full[2], out_ready[2], d_full[2], d_empty[2], y_full, x_ready, consts,
// drain, x_read) and the tensor-memory base address
constexpr int kOffTables = 2 * kTcSlotBytes;
constexpr int kNumBars = 13;
template <bool kInverse>
struct Tc5Layout {
  static constexpr int kTiles = kInverse ? kTc5InvTiles : kTc5FwdTiles;
  static constexpr int kFirstTile = kInverse ? 0 : kTc5InvTiles;
  static constexpr int kTableBytes = kTiles * kTc5TileBytes;
  static constexpr int kOffBars = kOffTables + kTableBytes;
  static constexpr int kOffTmemSlot = kOffBars + 8 * kNumBars;
  static constexpr int kSmemBytes = kOffTmemSlot + 8 + 1024;  // + slack to align the base
  static_assert(2 * kSmemBytes > 228 * 1024, "one CTA per SM: it owns all tensor memory");
  static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");
};
// tensor memory
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kColY = 0;
constexpr uint32_t kColD0 = 256;  // accumulator buffer b at kColD0 + 128 b
// instruction descriptors of kind::i8: D format s32 (bits 4-5 = 2), A / B
// format (bits 7-9 / 10-12: 0 unsigned, 1 signed), K-major A and B, N >> 3
// (bits 17-22) = 4, M >> 4 (bits 24-28) = 8: M = 128, N = 32, K = 32.
constexpr uint32_t kIdescU8 = (2u << 4) | (4u << 17) | (8u << 24);
constexpr uint32_t kIdescS8 = kIdescU8 | (1u << 7) | (1u << 10);
constexpr uint64_t kWaitNs = 2000000000ull;
// The first stage's sums S (in [-16 * 128 (q-1), 16 * 382 (q-1)]: unsigned
// low bytes and signed high bytes against constants below q) plus this
// multiple of q are non-negative and below 2^25: bytes 0-2 and a top byte of
// 0 or 1, all unsigned for the second stage.
constexpr uint32_t kFirstBias = 2048u * 3329u;

__device__ __align__(128) uint8_t g_tc5_tables[kTc5TableBytes];

// Shared-memory matrix descriptor (sm_100 format: start, leading and stride
// byte offsets in 16-byte units, version 1 at bit 46, layout at bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
constexpr uint32_t kLayoutNone = 0, kLayoutSw128 = 2;

__device__ __forceinline__ void st_shared_v2(uint32_t addr, uint32_t a, uint32_t b) {
  asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(addr), "r"(a), "r"(b) : "memory");
}
__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c,
                                             uint32_t d) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}
__device__ __forceinline__ uint4 ld_shared_v4(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(addr)
               : "memory");
  return v;
}

struct Tc5Params {
  CUtensorMap in;   // [npoly][256] uint16, boxes 64 x 128 rows, 128-byte swizzle
  CUtensorMap out;  // the same for the output (equal to in for in place)
  const uint8_t* tables;  // this direction's constant tiles (device copy)
  unsigned* status;
  int ntiles;
};

// Address of row p's 16-byte chunk k (0..31: bytes 16k .. 16k+15 of the
// natural 512-byte row) in a slot holding the TMA layout: quarter k / 8,
// rows 128 bytes apart, chunk index xor (p % 8) (the 128-byte swizzle).
__device__ __forceinline__ uint32_t sw128_chunk(uint32_t slot, uint32_t p, uint32_t k) {
  return slot + (k >> 3) * kTcQuarterBytes + p * 128u + (((k & 7u) ^ (p & 7u)) << 4);
}

// The forward's transposition: for coefficient c (c-tile c, 4 KiB at 4096 c
// of the slot), row p's 32 K bytes are the blocks' values X[m][c] in block
// order (K byte 2m + b), K-major without swizzle (8-row core matrices of
// 16-byte rows, the two K halves 128 bytes apart, 8-row groups 256 bytes
// apart).  Warp w reads coefficients 8 (w / 4) .. + 7 of every block of its
// rows, the 8 warps meet on an mbarrier (bounded wait), then every warp writes
// its c-tiles over the rows.  Stage 1 runs per c-tile in chunks of c-tiles
// {0-3}, {4-7}, ..., stage 2 per block i from tensor-memory columns 16 i ..
// 16 i + 15 against the block's own constant tiles, chunks of blocks {0-3},
// {4-7}, ...; its rows (two 16-byte chunks per block) go to the slot in the
// TMA layout.
template <bool kInverse>
__global__ void __launch_bounds__(kTcThreads, 1) k_tc5(const __grid_constant__ Tc5Params P) {
  using L = Tc5Layout<kInverse>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* const basep = smem_raw + (base - raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = (int)gridDim.x;
  const int t_begin = (int)((long long)blockIdx.x * P.ntiles / G);
  const int t_end = (int)((long long)(blockIdx.x + 1) * P.ntiles / G);
  const int nmine = t_end - t_begin;

  const uint32_t tables = base + kOffTables;
  const uint32_t bars = base + L::kOffBars;
  auto in_full = [&](int s) { return bars + 8u * s; };
  auto out_ready = [&](int s) { return bars + 16u + 8u * s; };
  auto d_full = [&](int b) { return bars + 32u + 8u * b; };
  auto d_empty = [&](int b) { return bars + 48u + 8u * b; };
  const uint32_t y_full = bars + 64u, x_ready = bars + 72u, consts = bars + 80u,
                 drain = bars + 88u, x_read = bars + 96u;
  auto slot_addr = [&](int s) { return base + (uint32_t)s * kTcSlotBytes; };

  if (tid == 0) {
    for (int s = 0; s < 2; s++) {
      mbar_init(in_full(s), 1);
      mbar_init(out_ready(s), kTcEpiWarps);
      mbar_init(d_full(s), 1);
      mbar_init(d_empty(s), 4);
    }
    mbar_init(y_full, kTcEpiWarps);
    mbar_init(x_ready, kTcEpiWarps);
    mbar_init(consts, 1);
    mbar_init(drain, 1);
    mbar_init(x_read, kTcEpiWarps);
    fence_mbar_init();
  }
  if (warp == kTcMmaWarp) {
    tmem_alloc(base + L::kOffTmemSlot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();  // the mbarriers are initialised (and fenced) before any use
  tc_fence_after();
  const uint32_t tmem = *(volatile uint32_t*)(basep + L::kOffTmemSlot);
  if (warp == kTcTmaWarp && lane == 0) {  // constant tiles (written once by the host)
    mbar_expect_tx(consts, L::kTableBytes);
    bulk_g2s(tables, P.tables, L::kTableBytes, consts);
  }
  // the tile data may have been written by the previous kernel in the stream
  grid_dependency_wait();
  grid_launch_dependents();

  bool ok = true;
  if (warp == kTcTmaWarp) {
    if (lane == 0) {
      // ---- producer: loads two tiles ahead, stores each tile's output ----
      int last_load[2] = {-1, -1};
      auto load = [&](int k, int s) {
        mbar_expect_tx(in_full(s), kTcSlotBytes);
        const int row = kTcTile * (t_begin + k);
        for (int q = 0; q < 4; q++)
          tma_load_2d(slot_addr(s) + q * kTcQuarterBytes, &P.in, 64 * q, row, in_full(s));
        last_load[s] = k;
      };
      for (int k = 0; k < 2 && k < nmine; k++) load(k, k);
      for (int k = 0; k < nmine; k++) {
        const int s = k & 1;
        if (!mbar_wait_bounded(out_ready(s), (uint32_t)(k >> 1) & 1u, kWaitNs)) {
          ok = false;
          break;
        }
        const int row = kTcTile * (t_begin + k);
        for (int q = 0; q < 4; q++)
          tma_store_2d(&P.out, 64 * q, row, slot_addr(s) + q * kTcQuarterBytes);
        bulk_commit();
        bulk_wait_read<0>();  // the slot may be refilled
        if (k + 2 < nmine) load(k + 2, s);
      }
      bulk_wait_all();
      // after a give-up: let issued loads land before the CTA's memory goes
      for (int s = 0; s < 2; s++)
        if (last_load[s] >= 0)
          ok &= mbar_wait_bounded(in_full(s), (uint32_t)(last_load[s] >> 1) & 1u, kWaitNs);
      ok &= mbar_wait_bounded(consts, 0, kWaitNs);
    }
  } else if (warp == kTcMmaWarp) {
    if (lane == 0 && nmine > 0) {
      // ---- MMA issuer ----
      auto tile_desc = [&](int i) {
        return smem_desc(tables + (uint32_t)(i - L::kFirstTile) * kTc5TileBytes, 128, 256,
                         kLayoutNone);
      };
      uint32_t use[2] = {0, 0};
      auto take = [&](int b) {  // the buffer's previous contents were read out
        if (use[b] > 0 && !mbar_wait_bounded(d_empty(b), (use[b] - 1) & 1u, kWaitNs))
          return false;
        tc_fence_after();
        return true;
      };
      ok = mbar_wait_bounded(consts, 0, kWaitNs);
      for (int k = 0; k < nmine && ok; k++) {
        const int s = k & 1;
        // inverse: the loaded tile is stage A's operand; forward: wait for
        // the epilogue warps' transposed copy of it
        if (kInverse)
          ok = mbar_wait_bounded(in_full(s), (uint32_t)(k >> 1) & 1u, kWaitNs);
        else
          ok = mbar_wait_bounded(x_ready, (uint32_t)k & 1u, kWaitNs);
        if (!ok) break;
        tc_fence_after();
        // first stage: chunk j = four MMA pairs (inverse: blocks 4j..4j+3 of
        // input quarter j; forward: c-tiles 4j..4j+3)
        for (int j = 0; j < 4 && ok; j++) {
          const int b = j & 1;
          if (!(ok = take(b))) break;
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int idx = 4 * j + u;
            const uint32_t d = tmem + kColD0 + 128u * b + 32u * u;
            if (kInverse) {
              const uint64_t a = smem_desc(slot_addr(s) + j * kTcQuarterBytes + 32 * u, 16, 1024,
                                           kLayoutSw128);
              tc_mma_ss(d, a, tile_desc(2 * idx), kIdescU8, 0);
              tc_mma_ss(d, a, tile_desc(2 * idx + 1), kIdescS8, 1);
            } else {
              const uint64_t a = smem_desc(slot_addr(s) + 4096u * idx, 128, 256, kLayoutNone);
              tc_mma_ss(d, a, tile_desc(34), kIdescU8, 0);
              tc_mma_ss(d, a, tile_desc(35), kIdescS8, 1);
            }
          }
          tc_commit(d_full(b));
          use[b]++;
        }
        if (!ok) break;
        // second stage from tensor memory: inverse coefficient sets {0-3},
        // {8-11}, {4-7}, {12-15}; forward blocks {0-3}, {4-7}, ...
        if (!(ok = mbar_wait_bounded(y_full, (uint32_t)k & 1u, kWaitNs))) break;
        tc_fence_after();
        for (int j = 0; j < 4 && ok; j++) {
          const int b = j & 1;
          if (!(ok = take(b))) break;
          // inverse: coefficient sets {0-3}, {8-11}, {4-7}, {12-15} (buffer 0,
          // warps 0-3: 0-7; buffer 1, warps 4-7: 8-15); forward: blocks 4j ..
          const int first = kInverse ? 8 * (j & 1) + 4 * (j >> 1) : 4 * j;
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int idx = first + u;
            const uint32_t d = tmem + kColD0 + 128u * b + 32u * u;
#pragma unroll
            for (int h = 0; h < 2; h++)
              tc_mma_ts(d, tmem + kColY + 16u * idx + 8u * h,
                        tile_desc(kInverse ? 32 + h : 36 + 2 * idx + h), kIdescU8, h);
          }
          tc_commit(d_full(b));
          use[b]++;
        }
      }
      // every MMA issued above has completed before tensor memory is freed
      tc_commit(drain);
      ok &= mbar_wait_bounded(drain, 0, kWaitNs);
    }
  } else {
    // ---- warps 0-7: tensor memory <-> registers <-> shared memory ----
    const int half = warp >> 2, lq = warp & 3;
    const uint32_t lanes = (uint32_t)(32 * lq) << 16;
    const uint32_t dcol = tmem + lanes + kColD0 + 128u * half;
    const uint32_t ycol = tmem + lanes + kColY;
    const uint32_t p = (uint32_t)(32 * lq + lane);  // polynomial (row) of the tile
    uint32_t use = 0;
    auto take = [&]() {
      const bool r = mbar_wait_bounded(d_full(half), use & 1u, kWaitNs);
      use++;
      tc_fence_after();
      return r;
    };
    auto give_back = [&]() {
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(d_empty(half));
    };
    for (int k = 0; k < nmine && ok; k++) {
      const int s = k & 1;
      const uint32_t slot = slot_addr(s);
      if (!kInverse) {
        // transpose the loaded tile in place into stage 1's operand
        const bool landed = mbar_wait_bounded(in_full(s), (uint32_t)(k >> 1) & 1u, kWaitNs);
        uint4 R[16];  // X[m][8 half .. 8 half + 7] as four coefficient pairs
#pragma unroll
        for (int m = 0; m < 16; m++) R[m] = ld_shared_v4(sw128_chunk(slot, p, 2u * m + half));
        // every warp's rows read before any c-tile is written over them
        __syncwarp();
        if (lane == 0) mbar_arrive(x_read);
        const bool read = mbar_wait_bounded(x_read, (uint32_t)k & 1u, kWaitNs);
        if (!__all_sync(0xffffffffu, landed && read)) {
          ok = false;
          break;
        }
#pragma unroll
        for (int cc = 0; cc < 8; cc++) {
          const uint32_t sel = (cc & 1) ? 0x7632u : 0x5410u;
          uint32_t w[8];
#pragma unroll
          for (int mp = 0; mp < 8; mp++) {
            const uint4 a = R[2 * mp], b = R[2 * mp + 1];
            const uint32_t wa = (cc >> 1) == 0 ? a.x : (cc >> 1) == 1 ? a.y : (cc >> 1) == 2 ? a.z : a.w;
            const uint32_t wb = (cc >> 1) == 0 ? b.x : (cc >> 1) == 1 ? b.y : (cc >> 1) == 2 ? b.z : b.w;
            w[mp] = __byte_perm(wa, wb, sel);
          }
          const uint32_t xa = slot + 4096u * (8u * half + cc) + (p >> 3) * 256u + (p & 7u) * 16u;
          st_shared_v4(xa, w[0], w[1], w[2], w[3]);
          st_shared_v4(xa + 128u, w[4], w[5], w[6], w[7]);
        }
        fence_proxy_async_smem();  // generic-proxy writes -> the tensor cores
        __syncwarp();
        if (lane == 0) mbar_arrive(x_ready);
      }
      // first stage: S = D_lo + 128 D_hi + 2048 q (non-negative, below 2^25)
      // as int32 to tensor memory column 16 n + idx (output n of the MMA,
      // idx = 4j + u its position among the tile's first-stage MMAs), the
      // second stage's K bytes 4 (idx % 8) .. + 3 of step idx / 8; chunks
      // j = half, half + 2
#pragma unroll 1
      for (int jj = 0; jj < 2; jj++) {
        const int j = half + 2 * jj;
        if (!__all_sync(0xffffffffu, take())) {
          ok = false;
          break;
        }
        uint32_t r0[64], r1[64];
        tc_ld64(dcol, r0);
        tc_ld64(dcol + 64, r1);
        tc_wait_ld();
        give_back();
#pragma unroll
        for (int n = 0; n < 16; n++)
          tc_st4(ycol + 16u * n + 4u * j, r0[n] + (r0[16 + n] << 7) + kFirstBias,
                 r0[32 + n] + (r0[48 + n] << 7) + kFirstBias,
                 r1[n] + (r1[16 + n] << 7) + kFirstBias, r1[32 + n] + (r1[48 + n] << 7) + kFirstBias);
      }
      if (!ok) break;
      tc_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(y_full);
      // second stage: reduce, pack, write the output rows into the slot
#pragma unroll 1
      for (int jj = 0; jj < 2; jj++) {
        const int j = half + 2 * jj;
        if (!__all_sync(0xffffffffu, take())) {
          ok = false;
          break;
        }
        if (kInverse) {
          // coefficients 16 i + c0 .. +3 of every block i (c0 = 8 half + 4 jj):
          // 8 bytes at byte 8 jj of 16-byte chunk 2 i + half
          uint32_t r0[64], r1[64];
          tc_ld64(dcol, r0);
          tc_ld64(dcol + 64, r1);
          tc_wait_ld();
          give_back();
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const uint32_t w0 = pack2(red_centred(r0[i] + (r0[16 + i] << 7)),
                                      red_centred(r0[32 + i] + (r0[48 + i] << 7)));
            const uint32_t w1 = pack2(red_centred(r1[i] + (r1[16 + i] << 7)),
                                      red_centred(r1[32 + i] + (r1[48 + i] << 7)));
            st_shared_v2(sw128_chunk(slot, p, 2u * i + half) + 8u * jj, w0, w1);
          }
        } else {
          uint32_t r0[64], r1[64];
          tc_ld64(dcol, r0);
          tc_ld64(dcol + 64, r1);
          tc_wait_ld();
          give_back();
          // blocks 4j .. 4j+3, each 16 coefficients = two 16-byte chunks
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const uint32_t* r = u < 2 ? r0 + 32 * u : r1 + 32 * (u - 2);
            uint32_t w[8];
#pragma unroll
            for (int t = 0; t < 8; t++)
              w[t] = pack2(red_exact(r[2 * t] + (r[16 + 2 * t] << 7)),
                           red_exact(r[2 * t + 1] + (r[17 + 2 * t] << 7)));
            const uint32_t i = 4u * j + u;
            st_shared_v4(sw128_chunk(slot, p, 2u * i), w[0], w[1], w[2], w[3]);
            st_shared_v4(sw128_chunk(slot, p, 2u * i + 1), w[4], w[5], w[6], w[7]);
          }
        }
      }
      if (!ok) break;
      fence_proxy_async_smem();  // generic-proxy writes -> the TMA store
      __syncwarp();
      if (lane == 0) mbar_arrive(out_ready(s));
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kTcMmaWarp) {
    __syncwarp();  // lane 0 issued the MMAs alone; dealloc is warp-wide
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
  if (!ok) atomicOr(P.status, kInverse ? 2u : 1u);
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
  });
  return fn;
}

// The batch as a [npoly][256] uint16 tensor: boxes of 64 coefficients x 128
// polynomials with the 128-byte swizzle (16 KiB each, four per tile).
bool encode_swizzled_map(CUtensorMap* map, const int16_t* base, int npoly) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encoder();
  if (!enc) {
    note_encode_result(-1);
    return false;
  }
  const cuuint64_t dims[2] = {256, (cuuint64_t)npoly};
  const cuuint64_t strides[1] = {512};
  const cuuint32_t box[2] = {64, (cuuint32_t)kTcTile};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, (void*)base, dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  note_encode_result((int)r);
  return r == CUDA_SUCCESS;
}

const uint8_t* g_tables_ptr[64];

}  // namespace

bool tc5_init_device(DeviceInfo* info) {
  static uint8_t image[kTc5TableBytes];
  static std::once_flag once;
  std::call_once(once, [] {
    static Matrices M;
    build_matrices(&M);
    build_tc5_tables(M, image);
  });
  if (info->device < 0 || info->device >= 64) return false;
  if (cudaMemcpyToSymbol(g_tc5_tables, image, sizeof(image)) != cudaSuccess) return false;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_tc5_tables) != cudaSuccess || !p) return false;
  g_tables_ptr[info->device] = (const uint8_t*)p;
  return cudaFuncSetAttribute((const void*)k_tc5<true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              Tc5Layout<true>::kSmemBytes) == cudaSuccess &&
         cudaFuncSetAttribute((const void*)k_tc5<false>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              Tc5Layout<false>::kSmemBytes) == cudaSuccess;
}

cudaError_t launch_tc5(bool inverse, const int16_t* src, int16_t* dst, long long npoly,
                       const DeviceInfo& info, cudaStream_t stream) {
  const uint8_t* tables = g_tables_ptr[info.device];
  if (!tables || !info.status) return cudaErrorInitializationError;
  const void* fn = inverse ? (const void*)k_tc5<true> : (const void*)k_tc5<false>;
  const int smem = inverse ? Tc5Layout<true>::kSmemBytes : Tc5Layout<false>::kSmemBytes;
  for (long long done = 0; done < npoly; done += kMaxLaunchPolys) {
    const int n = (int)((npoly - done) < kMaxLaunchPolys ? (npoly - done) : kMaxLaunchPolys);
    Tc5Params m = {};
    if (!encode_swizzled_map(&m.in, src + done * 256, n)) return cudaErrorInvalidResourceHandle;
    if (src == dst)
      m.out = m.in;
    else if (!encode_swizzled_map(&m.out, dst + done * 256, n))
      return cudaErrorInvalidResourceHandle;
    m.tables = tables + (inverse ? 0 : kTc5InvTiles * kTc5TileBytes);
    m.status = info.status;
    m.ntiles = (n + kTcTile - 1) / kTcTile;
    const int ctas = m.ntiles < info.num_sms ? m.ntiles : info.num_sms;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3((unsigned)kTcThreads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[1] = {(void*)&m};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace tk
