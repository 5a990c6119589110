// tk_tc5.cu -- batched ML-KEM inverse NTT on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, int32 accumulators in tensor memory), sm_100a.
//
// Same transform as the mma.sync inverse (tk_ntt_mma.cu) and the same method
// (TensorKyber's intt_core, ntt_bench/ntt_kernels.cuh:548-625): stage A
// applies the per-block matrices MA^(m) (Gentleman-Sande layers len 2..8),
// stage B the 16x16 matrix Minv over the block index m (layers len 16..128
// and the final x1441 Montgomery factor), every constant as two 7-bit int8
// limbs.  The B200 formulation:
//
//   * A tile is 128 polynomials, the M dimension of every MMA (one polynomial
//     per tensor-memory lane).  TMA loads it as four boxes of 64 coefficients
//     x 128 rows with the 128-byte swizzle, which is exactly the canonical
//     K-major SW128 operand layout: stage A's A operand for block m is the
//     32 bytes of that block in each row, read straight from the loaded tile.
//   * Signed data need no CUDA-core pass.  An int16 x = b0 + 256 b1 with b0
//     unsigned and b1 signed, so stage A is two MMAs per block into the same
//     accumulator: one with unsigned data and constants on the low bytes'
//     K rows (MA), one with signed data and constants on the high bytes' K rows
//     (256 MA mod q); the other rows of each constant tile are zero.
//   * Stage A's accumulators (lo / hi constant limb) are combined into the
//     int32 sum S = D_lo + 128 D_hi (one IMAD) and written back to tensor
//     memory transposed: column 16 c + m holds S of block m, coefficient c.
//     Stage B's A operand for coefficient c is then columns 16 c .. 16 c + 15
//     straight from tensor memory (K byte 4 (m - 8h) + j = byte j of S[m]),
//     again split in two MMA kinds: bytes 0-2 unsigned, byte 3 signed, so S is
//     taken exactly as two's complement and never reduced in between.
//   * Stage B's sums S (in [-2^16, 2^26)) get one centred exact reduction and
//     are packed to int16, written in the same swizzled layout over the tile's
//     own input slot (its MMAs have finished), and TMA stores the tile.
//
// Roles (320 threads, one CTA per SM by shared memory): warp 9 lane 0 issues
// TMA loads and stores; warp 8 lane 0 issues MMAs (and warp 8 owns the
// tensor-memory allocation); warps 0-7 move data between tensor memory,
// registers and shared memory, warps w and w + 4 sharing tensor-memory lanes
// 32 (w % 4) .. + 31 (polynomials) and splitting the columns.  Tensor memory
// (512 columns): 0-255 the transposed stage-A sums, 256-383 and 384-511 two
// accumulator buffers of four 32-column MMA results each.  Per tile the MMA
// thread issues 8 chunks (stage A blocks 0-3, 4-7, 8-11, 12-15, then stage B
// coefficient sets {0-3}, {8-11}, {4-7}, {12-15}) into the buffers in turn;
// warps 0-3 take buffer 0, warps 4-7 buffer 1.  Two input slots of 64 KiB:
// the load of tile k + 2 goes into tile k's slot once tile k's output
// (written over its input) has been read out by the store.  Every mbarrier
// wait gives up after 2 s (status bit 1, as the other inverse kernels); the
// MMA thread then drains its MMAs and the producer its copies before the
// CTA frees tensor memory and exits.
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
// dynamic shared memory, from a 1024-byte aligned base (the swizzle atom)
constexpr int kOffTables = 2 * kTcSlotBytes;
constexpr int kOffBars = kOffTables + kTc5TableBytes;
// in_full[2], out_ready[2], d_full[2], d_empty[2], y_full, consts, drain
constexpr int kNumBars = 11;
constexpr int kOffTmemSlot = kOffBars + 8 * kNumBars;
constexpr int kTcSmemUsed = kOffTmemSlot + 8;
constexpr int kTcSmemBytes = kTcSmemUsed + 1024;  // + slack to align the base
static_assert(2 * kTcSmemBytes > 228 * 1024, "one CTA per SM: it owns all tensor memory");
static_assert(kTcSmemBytes <= 227 * 1024, "shared memory per CTA");
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
// centred reduction of stage B's sums (red_centred_wide below)
constexpr int64_t kM40 = 330282857;  // ceil(2^40 / q) = floor(2^40 / q) + 1
constexpr int64_t kAdd40 = (3329ll * 65536 + 1664) * kM40;

__device__ __align__(128) uint8_t g_tc5_tables[kTc5TableBytes];

// Shared-memory matrix descriptor (sm_100 format: start, leading and stride
// byte offsets in 16-byte units, version 1 at bit 46, layout at bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
constexpr uint32_t kLayoutNone = 0, kLayoutSw128 = 2;

// S in [-2^16, 2^26): an int32 whose low 16 bits are the centred residue of S
// in [-(q-1)/2, (q-1)/2].  T = S + q 2^16 (a multiple of q and of 2^16) lies
// in [0, 2^28); floor((T + (q-1)/2) / q) = ((T + 1664) ceil(2^40/q)) >> 40
// exactly there (the multiplier's error adds < 2^28 / 2^40 < 1/q), as one
// 64-bit multiply-add; S - q quot differs from T - q quot by q 2^16.
__device__ __forceinline__ uint32_t red_centred_wide(uint32_t s) {
  const int64_t x = (int64_t)(int32_t)s * kM40 + kAdd40;
  const uint32_t quot = (uint32_t)((uint64_t)x >> 40);
  return s - quot * 3329u;
}

__device__ __forceinline__ void st_shared_v2(uint32_t addr, uint32_t a, uint32_t b) {
  asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(addr), "r"(a), "r"(b) : "memory");
}

struct Tc5Params {
  CUtensorMap in;   // [npoly][256] uint16, boxes 64 x 128 rows, 128-byte swizzle
  CUtensorMap out;  // the same for the output (equal to in for in place)
  const uint8_t* tables;
  unsigned* status;
  int ntiles;
};

__global__ void __launch_bounds__(kTcThreads, 1) k_invntt_tc5(const __grid_constant__ Tc5Params P) {
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
  const uint32_t bars = base + kOffBars;
  auto in_full = [&](int s) { return bars + 8u * s; };
  auto out_ready = [&](int s) { return bars + 16u + 8u * s; };
  auto d_full = [&](int b) { return bars + 32u + 8u * b; };
  auto d_empty = [&](int b) { return bars + 48u + 8u * b; };
  const uint32_t y_full = bars + 64u, consts = bars + 72u, drain = bars + 80u;
  auto slot_addr = [&](int s) { return base + (uint32_t)s * kTcSlotBytes; };

  if (tid == 0) {
    for (int s = 0; s < 2; s++) {
      mbar_init(in_full(s), 1);
      mbar_init(out_ready(s), kTcEpiWarps);
      mbar_init(d_full(s), 1);
      mbar_init(d_empty(s), 4);
    }
    mbar_init(y_full, kTcEpiWarps);
    mbar_init(consts, 1);
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == kTcMmaWarp) {
    tmem_alloc(base + kOffTmemSlot, kTmemCols);
    tmem_relinquish();
  }
  if (warp == kTcTmaWarp && lane == 0) {  // constant tiles (written once by the host)
    mbar_expect_tx(consts, kTc5TableBytes);
    bulk_g2s(tables, P.tables, kTc5TableBytes, consts);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *(volatile uint32_t*)(basep + kOffTmemSlot);
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
        return smem_desc(tables + (uint32_t)i * kTc5TileBytes, 128, 256, kLayoutNone);
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
        if (!(ok = mbar_wait_bounded(in_full(s), (uint32_t)(k >> 1) & 1u, kWaitNs))) break;
        tc_fence_after();
        // stage A: chunk j = blocks 4j .. 4j+3 (input quarter j)
        for (int j = 0; j < 4 && ok; j++) {
          const int b = j & 1;
          if (!(ok = take(b))) break;
#pragma unroll
          for (int mm = 0; mm < 4; mm++) {
            const int m = 4 * j + mm;
            const uint64_t a =
                smem_desc(slot_addr(s) + j * kTcQuarterBytes + 32 * mm, 16, 1024, kLayoutSw128);
            const uint32_t d = tmem + (kColD0 + 128u * b) + 32u * mm;
            tc_mma_ss(d, a, tile_desc(2 * m), kIdescU8, 0);
            tc_mma_ss(d, a, tile_desc(2 * m + 1), kIdescS8, 1);
          }
          tc_commit(d_full(b));
          use[b]++;
        }
        if (!ok) break;
        // stage B: coefficient sets {0-3}, {8-11}, {4-7}, {12-15}
        if (!(ok = mbar_wait_bounded(y_full, (uint32_t)k & 1u, kWaitNs))) break;
        tc_fence_after();
        for (int j = 0; j < 4 && ok; j++) {
          const int b = j & 1;
          if (!(ok = take(b))) break;
          const int c0 = 8 * (j & 1) + 4 * (j >> 1);
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const uint32_t d = tmem + (kColD0 + 128u * b) + 32u * u;
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const uint32_t a = tmem + kColY + 16u * (c0 + u) + 8u * h;
              tc_mma_ts(d, a, tile_desc(32 + 2 * h), kIdescU8, h);
              tc_mma_ts(d, a, tile_desc(33 + 2 * h), kIdescS8, 1);
            }
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
    const uint32_t dcol = tmem + lanes + (kColD0 + 128u * half);
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
      // stage A chunks j = half, half + 2: S[m][c] -> column 16 c + m
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
        for (int c = 0; c < 16; c++)
          tc_st4(ycol + 16u * c + 4u * j, r0[c] + (r0[16 + c] << 7), r0[32 + c] + (r0[48 + c] << 7),
                 r1[c] + (r1[16 + c] << 7), r1[32 + c] + (r1[48 + c] << 7));
      }
      if (!ok) break;
      tc_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(y_full);
      // stage B chunks: coefficients c0 .. c0+3 of every block i
      const uint32_t slot = slot_addr(s);
#pragma unroll 1
      for (int jj = 0; jj < 2; jj++) {
        const int j = half + 2 * jj;
        const int c0 = 8 * (j & 1) + 4 * (j >> 1);
        if (!__all_sync(0xffffffffu, take())) {
          ok = false;
          break;
        }
        uint32_t r0[64], r1[64];
        tc_ld64(dcol, r0);
        tc_ld64(dcol + 64, r1);
        tc_wait_ld();
        give_back();
        // row p, coefficients 16 i + c0 .. +3: 8 bytes at byte 32 (i % 4) +
        // 2 c0 of quarter i / 4, 16-byte chunk index xor (p % 8) (the swizzle)
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const uint32_t z0 = red_centred_wide(r0[i] + (r0[16 + i] << 7));
          const uint32_t z1 = red_centred_wide(r0[32 + i] + (r0[48 + i] << 7));
          const uint32_t z2 = red_centred_wide(r1[i] + (r1[16 + i] << 7));
          const uint32_t z3 = red_centred_wide(r1[32 + i] + (r1[48 + i] << 7));
          const uint32_t chunk = 2u * (i & 3) + (uint32_t)(c0 >> 3);
          const uint32_t addr = slot + (uint32_t)(i >> 2) * kTcQuarterBytes + p * 128u +
                                ((chunk ^ (p & 7u)) << 4) + 8u * ((uint32_t)(c0 >> 2) & 1u);
          st_shared_v2(addr, pack2(z0, z1), pack2(z2, z3));
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
  if (!ok) atomicOr(P.status, 2u);
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
  return cudaFuncSetAttribute((const void*)k_invntt_tc5,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kTcSmemBytes) == cudaSuccess;
}

cudaError_t launch_invntt_tc5(const int16_t* src, int16_t* dst, long long npoly,
                              const DeviceInfo& info, cudaStream_t stream) {
  const uint8_t* tables = g_tables_ptr[info.device];
  if (!tables || !info.status) return cudaErrorInitializationError;
  for (long long done = 0; done < npoly; done += kMaxLaunchPolys) {
    const int n = (int)((npoly - done) < kMaxLaunchPolys ? (npoly - done) : kMaxLaunchPolys);
    Tc5Params m = {};
    if (!encode_swizzled_map(&m.in, src + done * 256, n)) return cudaErrorInvalidResourceHandle;
    if (src == dst)
      m.out = m.in;
    else if (!encode_swizzled_map(&m.out, dst + done * 256, n))
      return cudaErrorInvalidResourceHandle;
    m.tables = tables;
    m.status = info.status;
    m.ntiles = (n + kTcTile - 1) / kTcTile;
    const int ctas = m.ntiles < info.num_sms ? m.ntiles : info.num_sms;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3((unsigned)kTcThreads);
    cfg.dynamicSmemBytes = (size_t)kTcSmemBytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[1] = {(void*)&m};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, (const void*)k_invntt_tc5, args);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace tk
