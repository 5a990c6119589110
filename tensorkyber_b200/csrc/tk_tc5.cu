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
//     loaded tile.  The forward contracts over m first, so the 16 epilogue
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
// Roles (608 threads, one CTA per SM by shared memory): warp 18 lane 0
// issues TMA loads and stores; lane 0 of warps 16 and 17 issue MMAs, warp
// 16 + j for the chunks of groups j and j + 2 (one issuing thread could not
// keep the tensor pipe fed: it shares its SMSP with busy epilogue warps), and
// warp 16 owns the tensor-memory allocation; warps 0-15 move data between
// tensor memory, registers and shared memory in four groups of four, warp w
// reaching tensor-memory lanes 32 (w % 4) .. + 31 (polynomials).  Tensor
// memory (512 columns): 0-255 the first stage's sums, 256 + 64 g .. + 63
// group g's accumulator buffer (two 32-column MMA results).  Per tile 16
// chunks of two results go out, chunk j into buffer j % 4, so the MMAs of one
// group's chunk run while the other groups read theirs, and the next tile's
// first stage starts while this tile's second-stage results are still being
// read (an mbarrier, y_free, keeps the next tile's sums from being written
// before both issuers' second-stage MMAs of this tile have read them).  The
// second stage's K step 0 reads only the sums of first-stage chunks 0-3,
// which the epilogue warps write first: a second mbarrier, y_half, lets each
// issuer start that step of its first two second-stage chunks while the other
// half of the sums is still being written.
// Three slots of 64 KiB: the load of tile k + 3 goes into tile k's slot once
// tile k's output (written over its input) has been read out by the store.
// Every mbarrier wait gives up after 2 s (status bit 0 forward / 1 inverse,
// as the other kernels); the issuers then drain their MMAs and the producer
// its copies before the CTA frees tensor memory and exits.
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
constexpr int kTcSlots = 3;
// epilogue warp groups: group g (warps 4g .. 4g + 3, one per tensor-memory
// lane quarter) owns accumulator buffer g
constexpr int kTcGroups = 4;
constexpr int kTcEpiWarps = 4 * kTcGroups;
// MMA issuers: warp kTcMmaWarp + j issues the chunks of groups j and j + 2
// (two SMSPs, so that no single thread has to keep the tensor pipe fed
// against the epilogue warps' instructions); the first also owns the TMEM
// allocation.  19 warps: registers are allocated for 20, 96 per thread.
constexpr int kTcIssuers = 2;
constexpr int kTcMmaWarp = kTcEpiWarps, kTcTmaWarp = kTcEpiWarps + kTcIssuers;
constexpr int kTcThreads = 32 * (kTcEpiWarps + kTcIssuers + 1);
// dynamic shared memory (its base is 1024-byte aligned, the swizzle atom;
// the kernel checks): three 64 KiB tile slots, this direction's constant
// tiles, the mbarriers (in_full[3], out_ready[3], d_full[4], d_empty[4],
// y_full, x_ready, x_read, consts, drain, y_free, y_half) and the
// tensor-memory base
// address
constexpr int kOffTables = kTcSlots * kTcSlotBytes;
constexpr int kNumBars = 2 * kTcSlots + 2 * kTcGroups + 7;
template <bool kInverse>
struct Tc5Layout {
  static constexpr int kTiles = kInverse ? kTc5InvTiles : kTc5FwdTiles;
  static constexpr int kFirstTile = kInverse ? 0 : kTc5InvTiles;
  static constexpr int kTableBytes = kTiles * kTc5TileBytes;
  static constexpr int kOffBars = kOffTables + kTableBytes;
  static constexpr int kOffTmemSlot = kOffBars + 8 * kNumBars;
  static constexpr int kSmemBytes = kOffTmemSlot + 8;
  static_assert(2 * kSmemBytes > 228 * 1024, "one CTA per SM: it owns all tensor memory");
  static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");
};
// tensor memory
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kColY = 0;
constexpr uint32_t kColD0 = 256;  // group g's accumulator buffer at kColD0 + 64 g
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

__device__ __forceinline__ void st_shared_u32(uint32_t addr, uint32_t a) {
  asm volatile("st.shared.u32 [%0], %1;" ::"r"(addr), "r"(a) : "memory");
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
__device__ __forceinline__ uint32_t word_of(const uint4& v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
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

// Per tile the two issuers send 16 chunks of two 32-column MMA results:
// first stage a = 0..7 (results 2a, 2a + 1: inverse blocks, forward
// coefficients), second stage b = 0..7 (results n = 4 (b % 4) + 2 (b / 4) and
// n + 1: inverse coefficients, forward blocks); chunk a or b goes to buffer
// (and warp group) a % 4 or b % 4, issued by issuer (a or b) % 2, so group g
// reads first-stage chunks g, g+4 and the second-stage results 4g .. 4g + 3.
// The MMAs of one chunk can run while the other groups read theirs.  The
// second stage's K step 0 waits for the first half of the sums in tensor
// memory (first-stage chunks 0-3, y_half), its K step 1 for all of them
// (y_full); the next tile's first stage waits only for its buffers.
//
// The forward's transposition: for coefficient c (c-tile c, 4 KiB at 4096 c
// of the slot), row p's 32 K bytes are the blocks' values X[m][c] in block
// order (K byte 2m + b), K-major without swizzle (8-row core matrices of
// 16-byte rows, the two K halves 128 bytes apart, 8-row groups 256 bytes
// apart).  The four warps of a lane quarter split each row: group g reads
// coefficients 8 (g % 2) .. + 7 of blocks 8 (g / 2) .. + 7 (eight 16-byte
// chunks), the 16 warps meet on an mbarrier (bounded wait), then every warp
// writes its half-K rows of c-tiles 8 (g % 2) .. + 7.  Tile k + 1 is
// transposed between tile k's two stages, while the second stage's first
// MMAs run.
template <bool kInverse>
__global__ void __launch_bounds__(kTcThreads, 1) k_tc5(const __grid_constant__ Tc5Params P) {
  using L = Tc5Layout<kInverse>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const uint32_t base = smem_u32(smem_raw);
  if (base & 1023u) {  // the swizzled slots need the 1024-byte atom alignment
    if (threadIdx.x == 0) atomicOr(P.status, kInverse ? 2u : 1u);
    return;
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = (int)gridDim.x;
  const int t_begin = (int)((long long)blockIdx.x * P.ntiles / G);
  const int t_end = (int)((long long)(blockIdx.x + 1) * P.ntiles / G);
  const int nmine = t_end - t_begin;

  const uint32_t tables = base + kOffTables;
  const uint32_t bars = base + L::kOffBars;
  auto in_full = [&](int s) { return bars + 8u * s; };
  auto out_ready = [&](int s) { return bars + 8u * (kTcSlots + s); };
  auto d_full = [&](int g) { return bars + 8u * (2 * kTcSlots + g); };
  auto d_empty = [&](int g) { return bars + 8u * (2 * kTcSlots + kTcGroups + g); };
  constexpr uint32_t kB = 8u * (2 * kTcSlots + 2 * kTcGroups);
  const uint32_t y_full = bars + kB, x_ready = bars + kB + 8u, x_read = bars + kB + 16u,
                 consts = bars + kB + 24u, drain = bars + kB + 32u, y_free = bars + kB + 40u,
                 y_half = bars + kB + 48u;
  auto slot_addr = [&](int s) { return base + (uint32_t)s * kTcSlotBytes; };

  if (tid == 0) {
    for (int s = 0; s < kTcSlots; s++) {
      mbar_init(in_full(s), 1);
      mbar_init(out_ready(s), kTcEpiWarps);
    }
    for (int g = 0; g < kTcGroups; g++) {
      mbar_init(d_full(g), 1);
      mbar_init(d_empty(g), 4);
    }
    mbar_init(y_full, kTcEpiWarps);
    mbar_init(x_ready, kTcEpiWarps);
    mbar_init(x_read, kTcEpiWarps);
    mbar_init(consts, 1);
    mbar_init(drain, kTcIssuers);
    mbar_init(y_free, kTcIssuers);
    mbar_init(y_half, kTcEpiWarps);
    fence_mbar_init();
  }
  if (warp == kTcMmaWarp) {  // the first issuer's warp
    tmem_alloc(base + L::kOffTmemSlot, kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();  // the mbarriers are initialised (and fenced) before any use
  tc_fence_after();
  const uint32_t tmem = *(volatile uint32_t*)(smem_raw + L::kOffTmemSlot);
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
      // ---- producer: loads three tiles ahead, stores each tile's output ----
      int last_load[kTcSlots];
      for (int s = 0; s < kTcSlots; s++) last_load[s] = -1;
      auto load = [&](int k) {
        const int s = k % kTcSlots;
        mbar_expect_tx(in_full(s), kTcSlotBytes);
        const int row = kTcTile * (t_begin + k);
        for (int q = 0; q < 4; q++)
          tma_load_2d(slot_addr(s) + q * kTcQuarterBytes, &P.in, 64 * q, row, in_full(s));
        last_load[s] = k;
      };
      for (int k = 0; k < kTcSlots && k < nmine; k++) load(k);
      for (int k = 0; k < nmine; k++) {
        const int s = k % kTcSlots;
        if (!mbar_wait_bounded(out_ready(s), (uint32_t)(k / kTcSlots) & 1u, kWaitNs)) {
          ok = false;
          break;
        }
        const int row = kTcTile * (t_begin + k);
        for (int q = 0; q < 4; q++)
          tma_store_2d(&P.out, 64 * q, row, slot_addr(s) + q * kTcQuarterBytes);
        bulk_commit();
        bulk_wait_read<0>();  // the slot may be refilled
        if (k + kTcSlots < nmine) load(k + kTcSlots);
      }
      bulk_wait_all();
      // after a give-up: let issued loads land before the CTA's memory goes
      for (int s = 0; s < kTcSlots; s++)
        if (last_load[s] >= 0)
          ok &= mbar_wait_bounded(in_full(s), (uint32_t)(last_load[s] / kTcSlots) & 1u, kWaitNs);
      ok &= mbar_wait_bounded(consts, 0, kWaitNs);
    }
  } else if (warp >= kTcMmaWarp) {
    if (lane == 0) {
      // ---- MMA issuer j: the chunks of groups j and j + 2 ----
      // Descriptors are built once (a shared-memory descriptor's low 14 bits
      // are the address / 16, so an operand at byte offset o is the base
      // descriptor + o / 16; every address here is below 2^18).
      const int j = warp - kTcMmaWarp;
      const uint64_t b_desc0 = smem_desc(tables, 128, 256, kLayoutNone);
      auto tile_desc = [&](int i) {
        return b_desc0 + (uint64_t)((i - L::kFirstTile) * (kTc5TileBytes >> 4));
      };
      const uint64_t a_desc0 = kInverse ? smem_desc(base, 16, 1024, kLayoutSw128)
                                        : smem_desc(base, 128, 256, kLayoutNone);
      // buffer g's previous contents were read out: every tile uses it four
      // times (first-stage chunks g, g + 4, second-stage chunks g, g + 4), so
      // the use at position pos (0..3) of tile k is use 4k + pos and waits
      // for the release of use 4k + pos - 1
      auto take = [&](int g, int k, int pos) {
        if ((k > 0 || pos > 0) && !mbar_wait_bounded(d_empty(g), (uint32_t)(pos + 1) & 1u, kWaitNs))
          return false;
        tc_fence_after();
        return true;
      };
      ok = mbar_wait_bounded(consts, 0, kWaitNs);
      for (int k = 0; k < nmine && ok; k++) {
        const int s = k % kTcSlots;
        // inverse: the loaded tile is stage A's operand; forward: wait for
        // the epilogue warps' transposed copy of it
        if (kInverse)
          ok = mbar_wait_bounded(in_full(s), (uint32_t)(k / kTcSlots) & 1u, kWaitNs);
        else
          ok = mbar_wait_bounded(x_ready, (uint32_t)k & 1u, kWaitNs);
        if (!ok) break;
        tc_fence_after();
        const uint64_t a_slot = a_desc0 + (uint64_t)(s * (kTcSlotBytes >> 4));
        // first stage: chunk a = g + 4 jj (g = j, j + 2) = results 2a, 2a + 1
        // (inverse: blocks; forward: c-tiles), an MMA pair each, both
        // results' first MMA before either second one; chunks in order a =
        // j, j + 2, j + 4, j + 6
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int g = j + 2 * (c & 1), jj = c >> 1, a = g + 4 * jj;
          if (!(ok = take(g, k, jj))) break;
          const uint32_t dbuf = tmem + kColD0 + 64u * (uint32_t)g;
#pragma unroll
          for (int t = 0; t < 2; t++)
#pragma unroll
            for (int u = 0; u < 2; u++) {
              const int idx = 2 * a + u;
              const uint64_t ad =
                  kInverse
                      ? a_slot + (uint64_t)(((idx >> 2) * kTcQuarterBytes + 32 * (idx & 3)) >> 4)
                      : a_slot + (uint64_t)((4096 * idx) >> 4);
              tc_mma_ss(dbuf + 32u * u, ad, tile_desc(kInverse ? 2 * idx + t : 34 + t),
                        t ? kIdescS8 : kIdescU8, t);
            }
          tc_commit(d_full(g));
        }
        if (!ok) break;
        // second stage from tensor memory, two K steps per result: chunk b =
        // g + 4 jj = results n = 4g + 2 jj, + 1.  K step h reads the sums of
        // first-stage chunks 4h .. 4h + 3, so step 0 of the chunks jj = 0
        // runs once that half is written (y_half), while the epilogue warps
        // are still writing the other half; the rest waits for y_full.
        auto b_mma = [&](int g, int jj, int h) {
          const uint32_t dbuf = tmem + kColD0 + 64u * (uint32_t)g;
#pragma unroll
          for (int u = 0; u < 2; u++) {
            const int n = 4 * g + 2 * jj + u;
            tc_mma_ts(dbuf + 32u * u, tmem + kColY + 16u * (uint32_t)n + 8u * h,
                      tile_desc(kInverse ? 32 + h : 36 + 2 * n + h), kIdescU8, h);
          }
        };
        if (!(ok = mbar_wait_bounded(y_half, (uint32_t)k & 1u, kWaitNs))) break;
        tc_fence_after();
#pragma unroll
        for (int c = 0; c < 2; c++) {
          if (!(ok = take(j + 2 * c, k, 2))) break;
          b_mma(j + 2 * c, 0, 0);
        }
        if (!ok) break;
        if (!(ok = mbar_wait_bounded(y_full, (uint32_t)k & 1u, kWaitNs))) break;
        tc_fence_after();
#pragma unroll
        for (int c = 0; c < 2; c++) {
          b_mma(j + 2 * c, 0, 1);
          tc_commit(d_full(j + 2 * c));
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
          if (!(ok = take(j + 2 * c, k, 3))) break;
          b_mma(j + 2 * c, 1, 0);
          b_mma(j + 2 * c, 1, 1);
          tc_commit(d_full(j + 2 * c));
        }
        if (!ok) break;
        // this issuer's reads of the first stage's sums are issued: the
        // barrier completes when both issuers' have finished, after which the
        // next tile's sums may be written over them
        tc_commit(y_free);
      }
      // every MMA issued above has completed before tensor memory is freed
      tc_commit(drain);
      ok &= mbar_wait_bounded(drain, 0, kWaitNs);
    }
  } else {
    // ---- warps 0-15: tensor memory <-> registers <-> shared memory ----
    const int g = warp >> 2, lq = warp & 3;
    const uint32_t lanes = (uint32_t)(32 * lq) << 16;
    const uint32_t dcol = tmem + lanes + kColD0 + 64u * g;
    const uint32_t ycol = tmem + lanes + kColY;
    const uint32_t p = (uint32_t)(32 * lq + lane);  // polynomial (row) of the tile
    uint32_t use = 0;
    auto take = [&]() {
      const bool r = mbar_wait_bounded(d_full(g), use & 1u, kWaitNs);
      use++;
      tc_fence_after();
      return __all_sync(0xffffffffu, r);
    };
    auto give_back = [&]() {
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(d_empty(g));
    };
    // forward: transpose tile t in place into stage 1's operand
    auto transpose = [&](int t) {
      const int s = t % kTcSlots;
      const uint32_t slot = slot_addr(s);
      const uint32_t mh = (uint32_t)g >> 1, ch = (uint32_t)g & 1u;
      const bool landed = mbar_wait_bounded(in_full(s), (uint32_t)(t / kTcSlots) & 1u, kWaitNs);
      uint4 R[8];  // X[8 mh + mm][8 ch .. 8 ch + 7] as four coefficient pairs
#pragma unroll
      for (int mm = 0; mm < 8; mm++)
        R[mm] = ld_shared_v4(sw128_chunk(slot, p, 2u * (8u * mh + mm) + ch));
      // every warp's rows read before any c-tile is written over them
      __syncwarp();
      if (lane == 0) mbar_arrive(x_read);
      const bool read = mbar_wait_bounded(x_read, (uint32_t)t & 1u, kWaitNs);
      if (!__all_sync(0xffffffffu, landed && read)) return false;
#pragma unroll
      for (int cc = 0; cc < 8; cc++) {
        const uint32_t sel = (cc & 1) ? 0x7632u : 0x5410u;
        uint32_t w[4];
#pragma unroll
        for (int mp = 0; mp < 4; mp++)
          w[mp] = __byte_perm(word_of(R[2 * mp], cc >> 1), word_of(R[2 * mp + 1], cc >> 1), sel);
        st_shared_v4(slot + 4096u * (8u * ch + cc) + (p >> 3) * 256u + (p & 7u) * 16u + 128u * mh,
                     w[0], w[1], w[2], w[3]);
      }
      fence_proxy_async_smem();  // generic-proxy writes -> the tensor cores
      __syncwarp();
      if (lane == 0) mbar_arrive(x_ready);
      return true;
    };
    for (int k = 0; k < nmine && ok; k++) {
      const int s = k % kTcSlots;
      const uint32_t slot = slot_addr(s);
      if (!kInverse && k == 0 && !transpose(0)) {
        ok = false;
        break;
      }
      // first stage: S = D_lo + 128 D_hi + 2048 q (non-negative, below 2^25)
      // as int32 to tensor memory column 16 n + idx (output n of result idx),
      // the second stage's K bytes 4 (idx % 8) .. + 3 of step idx / 8.  The
      // previous tile's second-stage MMAs (from every issuer) read these
      // columns: y_free says they have finished.
#pragma unroll 1
      for (int jj = 0; jj < 2; jj++) {
        const uint32_t a = (uint32_t)g + 4u * jj;
        if (!take() ||
            (jj == 0 && k > 0 &&
             !__all_sync(0xffffffffu, mbar_wait_bounded(y_free, (uint32_t)(k - 1) & 1u, kWaitNs)))) {
          ok = false;
          break;
        }
        if (jj == 0 && k > 0) tc_fence_after();
        uint32_t r[64];
        tc_ld64_sync(dcol, r);
        give_back();
#pragma unroll
        for (int n = 0; n < 16; n++)
          tc_st2(ycol + 16u * n + 2u * a, r[n] + (r[16 + n] << 7) + kFirstBias,
                 r[32 + n] + (r[48 + n] << 7) + kFirstBias);
        if (jj == 0) {
          // the sums of first-stage chunks 0-3 (columns 16 n .. 16 n + 7,
          // the second stage's K step 0) are written once all 16 warps arrive
          tc_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(y_half);
        }
      }
      if (!ok) break;
      tc_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(y_full);
      if (!kInverse && k + 1 < nmine && !transpose(k + 1)) {
        ok = false;
        break;
      }
      // second stage: reduce, pack, write the output rows over the tile's
      // own slot (its first-stage MMAs have completed)
      if (kInverse) {
        // results 4g .. 4g + 3 = coefficients 16 i + 4g .. + 3 of every
        // block i, two per chunk.  Each chunk's pair is stored as soon as it
        // is reduced: a build that kept the first chunk's packed words in
        // registers across the wait for the second chunk stored the second
        // chunk's words in both halves.
#pragma unroll 1
        for (int jj = 0; jj < 2; jj++) {
          if (!take()) {
            ok = false;
            break;
          }
          uint32_t r[64];
          tc_ld64_sync(dcol, r);
          give_back();
          // coefficients 16 i + 4g + 2jj, + 1: 4 bytes at byte 8 (g % 2) +
          // 4 jj of 16-byte chunk 2i + g / 2
          const uint32_t off = 8u * (g & 1) + 4u * jj;
#pragma unroll
          for (int i = 0; i < 16; i++)
            st_shared_u32(sw128_chunk(slot, p, 2u * i + ((uint32_t)g >> 1)) + off,
                          pack2(red_centred(r[i] + (r[16 + i] << 7)),
                                red_centred(r[32 + i] + (r[48 + i] << 7))));
        }
      } else {
        // results = blocks 4g + 2jj, + 1, each 16 coefficients = two 16-byte
        // chunks
#pragma unroll 1
        for (int jj = 0; jj < 2; jj++) {
          if (!take()) {
            ok = false;
            break;
          }
          uint32_t r[64];
          tc_ld64_sync(dcol, r);
          give_back();
#pragma unroll
          for (int u = 0; u < 2; u++) {
            const uint32_t* ru = r + 32 * u;
            uint32_t w[8];
#pragma unroll
            for (int t = 0; t < 8; t++)
              w[t] = pack2(red_exact(ru[2 * t] + (ru[16 + 2 * t] << 7)),
                           red_exact(ru[2 * t + 1] + (ru[17 + 2 * t] << 7)));
            const uint32_t i = 4u * g + 2u * jj + u;
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
    __syncwarp();  // lane 0 issued MMAs alone; dealloc is warp-wide
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
