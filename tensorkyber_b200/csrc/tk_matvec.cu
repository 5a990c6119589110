// tk_matvec.cu -- batched ML-KEM matrix-vector jobs
//     out_i = invntt( sum_j basemul(A_ij, ntt(s_j)) ) + e_i,   i, j < k,
// the composition of the reference's ntt (ntt_bench/ref/ntt.c:80-95), basemul
// (ntt_bench/ref/ntt.c:139-146, applied pairwise as in ML-KEM's
// poly_basemul_montgomery) and invntt (ntt_bench/ref/ntt.c:106-126); the
// reference repository has no polyvec layer, so tko_matvec_job in the oracle
// restates the composition (barrett of the k-term sum before invntt, as ML-KEM's
// polyvec_basemul_acc_montgomery does).
//
// Execution, in chunks of jobs whose vectors fit in L2 (a chunk draws jobs
// from all uniform-k batches of the call, one piece per batch):
//   1. forward NTT  s -> out           (k_ntt_mma, out of place, all pieces in
//                                       one launch)
//   2. basemul-acc  out <- A o out     (k_basemul_acc<k>, in place per job, one
//                                       launch per piece)
//   3. inverse NTT  out -> out + e     (k_ntt_mma with addend, one launch)
// Steps 2 and 3 read the previous step's output from L2 (a chunk holds a
// bounded number of vector polynomials), so HBM sees A, s and e read once and out
// written once, the traffic of a single fused kernel, and no scratch memory
// is used.  All launches are stream-ordered (programmatic dependent launch),
// so a whole call can be captured into one CUDA graph.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "tk_internal.h"
#include "tk_ptx.cuh"
#include "tk_stages.cuh"
#include "tk_tables.h"

namespace tk {

// Pair constants z_t * 2^-16 mod q (build_pair_constants).
__device__ int32_t g_bm_zr[128];

constexpr uint32_t kAccBias = 1073742318u;    // q * ceil(2^30 / q)

__device__ __forceinline__ uint32_t mulmod_lazy(uint32_t x, uint32_t c) {
  return red_lazy(x * c);  // x < q + 8, c < q: x * c < 2^24
}

// One warp per job; lane l owns coefficient pairs 4l .. 4l+3 (16 bytes of every
// polynomial).  vec holds ntt(s) on entry and the accumulated products on
// exit.  All k + k^2 loads of a job are issued before any arithmetic (the
// kernel streams A from HBM and is bound by loads in flight); the products
// are accumulated as in basemul_row.
template <int K>
__global__ void __launch_bounds__(256) k_basemul_acc(const int16_t* __restrict__ A,
                                                     int16_t* __restrict__ vec, int njobs) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  uint32_t zr[4];
#pragma unroll
  for (int u = 0; u < 4; u++) zr[u] = (uint32_t)g_bm_zr[4 * lane + u];
  grid_dependency_wait();
  grid_launch_dependents();
  for (int job = gw; job < njobs; job += nw) {
    uint4 b[K], a[K][K];
#pragma unroll
    for (int j = 0; j < K; j++)
      b[j] = *(const uint4*)(vec + ((size_t)job * K + j) * 256 + 8 * lane);
#pragma unroll
    for (int i = 0; i < K; i++)
#pragma unroll
      for (int j = 0; j < K; j++)
        a[i][j] = __ldcs((const uint4*)(A + (((size_t)job * K + i) * K + j) * 256 + 8 * lane));
#pragma unroll
    for (int i = 0; i < K; i++)
      *(uint4*)(vec + ((size_t)job * K + i) * 256 + 8 * lane) = basemul_row<K>(a[i], b, zr);
  }
}

static bool upload_pair_constants() {
  int32_t zr[128];
  build_pair_constants(zr);
  return cudaMemcpyToSymbol(g_bm_zr, zr, sizeof(zr)) == cudaSuccess;
}

// ============================================================================
// Fused single-launch form: one warp runs a whole job, forward NTT of s,
// basemul-accumulate, inverse NTT plus e, in an 8-row padded smem buffer (rows
// >= k hold stale data; their results are never stored).  The per-block
// constants of both block-wise stages sit in CTA-shared smem, the stage-over-m
// constants and the pair constants in registers.  Used for the single-launch
// matvec mode and by the serving loop (tk_serve.cu).
// ============================================================================
__device__ FwdFrags g_mv_fwd;
__device__ InvFrags g_mv_inv;

// smem constants, per block pair P (blocks 2P, 2P+1), block h of the pair and
// lane: 4 words of fragments (parity even, odd; 2 words each), and for the
// inverse 4 accumulator-init words per lane.
struct FusedConsts {
  uint32_t fwd[8][2][32][4];  // [pair][block of the pair][lane]: 16 B per lane,
  uint32_t inv[8][2][32][4];  // lanes 16 B apart (conflict-free 128-bit loads)
  int32_t inv_c[8][32][4];
};
constexpr int kFusedConstBytes = (int)sizeof(FusedConsts);

__device__ __forceinline__ void fused_load_consts(FusedConsts* C) {
  for (int idx = threadIdx.x; idx < 8 * 32; idx += blockDim.x) {
    const int P = idx >> 5, lane = idx & 31;
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int sp = 0; sp < 2; sp++) {
        const int b = 2 * P + h;
#pragma unroll
        for (int j = 0; j < 2; j++) {
          C->fwd[P][h][lane][2 * sp + j] = g_mv_fwd.s2[b][sp][lane][j];
          C->inv[P][h][lane][2 * sp + j] = g_mv_inv.sa[b][sp][lane][j];
        }
        C->inv_c[P][lane][2 * h + sp] = g_mv_inv.ca[b][sp][lane];
      }
  }
}

struct WarpRegs {
  uint32_t am_f[2][4], am_i[2][4];
  int32_t c1lo, c1hi;
  uint32_t zr[4];
};

// Global loads of a job's inputs.  kLoad 0: streaming (__ldcs, tk_matvec);
// 1: volatile (__ldcv, the serving loop).  Serving inputs are either pool
// memory reused by later requests or a caller's pinned host buffers read in
// place, whose contents the host may rewrite between requests while the loop
// keeps running: ld.cv never returns a stale L1 line, and for system memory
// it discards a matching L2 line and fetches again.
template <int kLoad>
__device__ __forceinline__ uint4 job_ld16(const void* p) {
  return kLoad ? __ldcv((const uint4*)p) : __ldcs((const uint4*)p);
}
template <int kLoad>
__device__ __forceinline__ uint32_t job_ld4(const void* p) {
  return kLoad ? __ldcv((const uint32_t*)p) : __ldcs((const uint32_t*)p);
}

// ng consecutive jobs of width k (2..4; ng * k <= 8) on this warp: their k*ng
// vector polynomials fill the rows of one 8-row tile, so the block-wise stages
// (which always run on 8 rows) are shared by the group.  A / s / e / out point
// at the group's first job; the jobs' data are consecutive.  rows/rowp: the
// warp's 8 x 528-byte buffer (smem address / pointer).
template <int kLoad>
__device__ __forceinline__ void fused_job(int k, int ng, const int16_t* __restrict__ A,
                                          const int16_t* __restrict__ s,
                                          const int16_t* __restrict__ e, int16_t* __restrict__ out,
                                          uint32_t rows, uint8_t* rowp, const FusedConsts* C,
                                          const WarpRegs& R, int lane) {
  const int q4 = lane & 3, g8 = lane >> 2;
  const uint32_t ldt_off = 32u * ((lane & 7) + 8 * ((lane >> 3) & 1)) + 16u * (lane >> 4);
  const uint32_t hb1 = (lane >> 4) & 1;
  const uint32_t w_even = 32u * g8 + 16u * hb1 + 4u * q4;
  const uint32_t w_odd = 32u * g8 + 16u * (hb1 ^ 1) + 4u * q4;
  const uint32_t w_nat = 32u * g8 + 4u * q4;
  const uint32_t row_l = kRowBytes * (lane & 7) + 32u * (lane >> 4);
  const uint32_t stc_off = kRowBytes * (2 * q4) + 4u * g8;
  const uint32_t zero_add[4] = {0, 0, 0, 0};

  const int nrows = k * ng;
  // 1. s -> rows (each lane moves 16 bytes of every polynomial)
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j < nrows) {
      const uint4 v = job_ld16<kLoad>(s + j * 256 + 8 * lane);
      *(uint4*)(rowp + j * kRowBytes + 16 * lane) = v;
    }
  __syncwarp();
  // 2. forward stage 1 (M1), x ^ 0x8000 bias, parity-split rows
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j < nrows) {
      uint32_t b[4];
      ldsm_x4_t(rows + j * kRowBytes + ldt_off, b[0], b[1], b[2], b[3]);
      stage_m<false>(R.am_f, R.c1lo, R.c1hi, b[0] ^ 0x80008000u, b[1] ^ 0x80008000u,
                     b[2] ^ 0x80008000u, b[3] ^ 0x80008000u, rowp + j * kRowBytes, w_even, w_odd,
                     0, zero_add);
    }
  __syncwarp();
  // 3. forward stage 2 (M2), all 8 block pairs on the 8-row n-tile
#pragma unroll 2
  for (int P = 0; P < 8; P++) {
    const uint32_t hbw = (P >> 1) & 1;
    uint32_t r[4];
    ldsm_x4(rows + 64u * P + row_l + 16u * (((lane >> 3) & 1) ^ hbw), r[0], r[1], r[2], r[3]);
    const uint4 f0 = *(const uint4*)&C->fwd[P][0][lane][0];
    const uint4 f1 = *(const uint4*)&C->fwd[P][1][lane][0];
    const uint32_t a[2][2][2] = {{{f0.x, f0.y}, {f0.z, f0.w}}, {{f1.x, f1.y}, {f1.z, f1.w}}};
    const int32_t zc[2][2] = {{0, 0}, {0, 0}};
    stage_c<false>(a, zc, r, rowp + 64 * P + stc_off);
  }
  __syncwarp();
  // 4. basemul-accumulate over j, job by job, accumulators in registers;
  // acc_i -> the job's row i (after all of the job's rows were read)
#pragma unroll 1
  for (int t = 0; t < ng; t++) {
  const int16_t* At = A + (size_t)t * k * k * 256;
  uint8_t* rt = rowp + t * k * kRowBytes;
  int32_t acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int u = 0; u < 4; u++) acc[i][u][0] = acc[i][u][1] = 0;
#pragma unroll
  for (int j = 0; j < 4; j++)
    if (j < k) {
      const uint4 v = *(const uint4*)(rt + j * kRowBytes + 16 * lane);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
      uint32_t B0[4], B1[4], Bz[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        B0[u] = mulmod_lazy(w[u] & 0xffffu, kRinv);
        B1[u] = mulmod_lazy(w[u] >> 16, kRinv);
        Bz[u] = mulmod_lazy(w[u] >> 16, R.zr[u]);
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (i < k) {
          const uint4 av = job_ld16<kLoad>(At + (i * k + j) * 256 + 8 * lane);
          const uint32_t aw[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int32_t a0 = (int16_t)(aw[u] & 0xffffu), a1 = (int32_t)aw[u] >> 16;
            acc[i][u][0] += a0 * (int32_t)B0[u] + a1 * (int32_t)Bz[u];
            acc[i][u][1] += a0 * (int32_t)B1[u] + a1 * (int32_t)B0[u];
          }
        }
    }
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (i < k) {
      uint32_t o[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        o[u] = pack2(red_wide((uint32_t)acc[i][u][0] + kAccBias),
                     red_wide((uint32_t)acc[i][u][1] + kAccBias));
      *(uint4*)(rt + i * kRowBytes + 16 * lane) = make_uint4(o[0], o[1], o[2], o[3]);
    }
  }
  __syncwarp();
  // 5. inverse stage A (MA), natural order in and out
#pragma unroll 2
  for (int P = 0; P < 8; P++) {
    uint32_t r[4];
    ldsm_x4(rows + 64u * P + row_l + 16u * ((lane >> 3) & 1), r[0], r[1], r[2], r[3]);
    const uint32_t x0 = r[0] ^ 0x80008000u, x1 = r[1] ^ 0x80008000u;
    const uint32_t x2 = r[2] ^ 0x80008000u, x3 = r[3] ^ 0x80008000u;
    const uint32_t x[4] = {__byte_perm(x0, x1, 0x5410), __byte_perm(x0, x1, 0x7632),
                           __byte_perm(x2, x3, 0x5410), __byte_perm(x2, x3, 0x7632)};
    const uint4 f0 = *(const uint4*)&C->inv[P][0][lane][0];
    const uint4 f1 = *(const uint4*)&C->inv[P][1][lane][0];
    const int4 cv = *(const int4*)&C->inv_c[P][lane][0];
    const uint32_t a[2][2][2] = {{{f0.x, f0.y}, {f0.z, f0.w}}, {{f1.x, f1.y}, {f1.z, f1.w}}};
    const int32_t ca[2][2] = {{cv.x, cv.y}, {cv.z, cv.w}};
    stage_c<true>(a, ca, x, rowp + 64 * P + stc_off);
  }
  __syncwarp();
  // 6. inverse stage B (Minv), centred, plus e
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j < nrows) {
      uint32_t add[4] = {0, 0, 0, 0};
      if (e) {
        const uint32_t* ew = (const uint32_t*)(e + j * 256) + 8 * g8 + q4;
        add[0] = job_ld4<kLoad>(ew);
        add[1] = job_ld4<kLoad>(ew + 4);
        add[2] = job_ld4<kLoad>(ew + 64);
        add[3] = job_ld4<kLoad>(ew + 68);
      }
      uint32_t b[4];
      ldsm_x4_t(rows + j * kRowBytes + ldt_off, b[0], b[1], b[2], b[3]);
      stage_m<true, true>(R.am_i, 0, 0, b[0], b[1], b[2], b[3], rowp + j * kRowBytes, 0, 0, w_nat,
                    add);
    }
  __syncwarp();
  // 7. rows -> out
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j < nrows) {
      const uint4 v = *(const uint4*)(rowp + j * kRowBytes + 16 * lane);
      __stcs((uint4*)(out + j * 256 + 8 * lane), v);
    }
  __syncwarp();
}

__device__ __forceinline__ void fused_warp_regs(WarpRegs& R, int lane) {
#pragma unroll
  for (int g = 0; g < 2; g++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      R.am_f[g][j] = g_mv_fwd.s1[g][lane][j];
      R.am_i[g][j] = g_mv_inv.sb[g][lane][j];
    }
  R.c1lo = g_mv_fwd.c1[lane][0];
  R.c1hi = g_mv_fwd.c1[lane][1];
#pragma unroll
  for (int u = 0; u < 4; u++) R.zr[u] = (uint32_t)g_bm_zr[4 * lane + u];
}

constexpr int kFusedWarps = 4;
constexpr int kFusedWarpBytes = 8 * kRowBytes;
constexpr int kFusedSmem = kFusedConstBytes + kFusedWarps * kFusedWarpBytes;

__global__ void __launch_bounds__(32 * kFusedWarps)
    k_matvec_fused(const __grid_constant__ FusedBatches args) {
  extern __shared__ __align__(128) uint8_t smem[];
  FusedConsts* C = (FusedConsts*)smem;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t* rowp = smem + kFusedConstBytes + warp * kFusedWarpBytes;
  const uint32_t rows = smem_u32(rowp);
  fused_load_consts(C);
  WarpRegs R;
  fused_warp_regs(R, lane);
  __syncthreads();
  grid_dependency_wait();
  grid_launch_dependents();
  // work items: groups of floor(8 / k) consecutive jobs of one batch
  const int total = args.gfirst[args.nb];
  const int gw = blockIdx.x * kFusedWarps + warp, nw = gridDim.x * kFusedWarps;
  for (int item = gw; item < total; item += nw) {
    int b = 0;
    while (b + 1 < args.nb && item >= args.gfirst[b + 1]) b++;
    const int k = args.k[b];
    const int per = 8 / k;
    const int j0 = (item - args.gfirst[b]) * per;
    const int njobs = args.first[b + 1] - args.first[b];
    const int ng = njobs - j0 < per ? njobs - j0 : per;
    const size_t t = (size_t)j0;
    fused_job<0>(k, ng, args.A[b] + t * k * k * 256, args.s[b] + t * k * 256,
                 args.e[b] ? args.e[b] + t * k * 256 : nullptr, args.out[b] + t * k * 256, rows,
                 rowp, C, R, lane);
  }
}

// ============================================================================
// Serving loop: a persistent kernel, one CTA of kServeWarps warps per SM, that
// claims published jobs from the device-resident ring, runs fused_job on them
// and counts completions per request; the warp that completes a request
// fences its outputs system-wide and writes the request's generation into the
// request's flag in mapped host memory.
//
// Job descriptors live in a ring in mapped page-locked host memory (written
// by the host, read here once per claimed job).  Claiming is per CTA.  An idle warp marks itself in s_idle and watches its
// shared-memory mailbox; one idle warp at a time (s_lock) acts as the CTA's
// poller: it reads the global head and tail and, while head < tail, claims
// min(idle warps, tail - head) jobs with one compare-and-swap on head and
// hands them to the idle warps' mailboxes (itself included).  An unpublished
// slot is never claimed, so the loop may stop at any idle point.  With one
// poller per SM the head line sees 148 pollers, not thousands of warps.
//
// Every wait is bounded.  The loop leaves as a whole: once no CTA has claimed
// a job for idle_ns (ctl->last_claim_ns) a poller sets ctl->closing, and
// every CTA's poller then tells its warps to leave (a warp finishes a claimed
// job first).  ctl->stop from the host ends it the same way.  The host clears
// closing before a relaunch.  Idle polling backs off from 128 ns to 2 us.
// ============================================================================
constexpr int kServeWarps = 16;

__device__ __forceinline__ uint4 shfl_u4(const uint4& v, int src) {
  return make_uint4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                    __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}
constexpr int kServeSmem = kFusedConstBytes + kServeWarps * kFusedWarpBytes;
constexpr unsigned long long kNoJob = ~0ull, kExitJob = ~0ull - 1;

__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__global__ void __launch_bounds__(32 * kServeWarps, 1)
    k_serve(const ServeJob* __restrict__ ring, uint32_t ring_mask, ServeCtl* ctl,
            unsigned int* req_ctr, unsigned int* req_flag, unsigned long long idle_ns) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ unsigned long long s_job[kServeWarps];  // mailbox: job, kNoJob or kExitJob
  __shared__ unsigned int s_idle;                    // warps waiting for a job
  __shared__ int s_lock, s_exit;
  FusedConsts* C = (FusedConsts*)smem;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t* rowp = smem + kFusedConstBytes + warp * kFusedWarpBytes;
  const uint32_t rows = smem_u32(rowp);
  if (threadIdx.x < kServeWarps) s_job[threadIdx.x] = kNoJob;
  if (threadIdx.x == 0) {
    s_idle = 0;
    s_lock = 0;
    s_exit = 0;
  }
  fused_load_consts(C);
  WarpRegs R;
  fused_warp_regs(R, lane);
  __syncthreads();
  const unsigned long long t_start = globaltimer_ns();
  volatile unsigned long long* box = &s_job[warp];
  while (true) {
    unsigned long long got = kNoJob;
    if (lane == 0) {
      atomicOr(&s_idle, 1u << warp);
      unsigned int backoff = 128;
      while (true) {
        const unsigned long long mine = *box;
        if (mine != kNoJob) {
          *box = kNoJob;
          got = mine;
          break;
        }
        if (atomicCAS(&s_lock, 0, 1) != 0) {  // another warp is polling
          __nanosleep(64);
          continue;
        }
        // this warp polls for the CTA
        bool claimed = false;
        if (*(volatile int*)&s_exit || ld_relaxed_u32(&ctl->closing) || ld_relaxed_u32(&ctl->stop)) {
          *(volatile int*)&s_exit = 1;
          *box = kExitJob;
        } else {
          const unsigned int h = ld_relaxed_u32(&ctl->head);
          unsigned int t;
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(t) : "l"(&ctl->tail) : "memory");
          const int avail = (int)(t - h);
          if (avail > 0) {
            const unsigned int idle = *(volatile unsigned int*)&s_idle;
            const int n = min(avail, __popc(idle));
            if (atomicCAS(&ctl->head, h, h + (unsigned)n) == h) {
              asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(&ctl->last_claim_ns),
                           "l"(globaltimer_ns())
                           : "memory");
              unsigned int m = idle, given = 0;
              for (int i = 0; i < n; i++) {
                const int w = __ffs(m) - 1;
                m &= m - 1;
                given |= 1u << w;
                ((volatile unsigned long long*)s_job)[w] = (unsigned long long)(h + (unsigned)i);
              }
              atomicAnd(&s_idle, ~given);
            }
            claimed = true;  // claimed, or lost the race: poll again at once
          } else {
            unsigned long long last;
            asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(last)
                         : "l"(&ctl->last_claim_ns)
                         : "memory");
            // signed: another SM's timer may run slightly ahead of this one's
            const long long since =
                (long long)(globaltimer_ns() - (last > t_start ? last : t_start));
            if (since > (long long)idle_ns) {
              asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(&ctl->closing), "r"(1u)
                           : "memory");
              *(volatile int*)&s_exit = 1;
              *box = kExitJob;
            }
          }
        }
        __threadfence_block();
        atomicExch(&s_lock, 0);
        if (!claimed && *box == kNoJob) {
          __nanosleep(backoff);
          if (backoff < 2048) backoff <<= 1;
        }
      }
      __threadfence_block();
    }
    got = __shfl_sync(0xffffffffu, got, 0);
    if (got == kExitJob) break;  // warp-uniform exit
    // the descriptor, from the ring in host memory: lanes 0..2 fetch its
    // 16-byte parts (uncached: the host rewrites entries as the ring wraps)
    uint4 part = make_uint4(0, 0, 0, 0);
    if (lane < 3) part = __ldcv((const uint4*)(ring + (got & ring_mask)) + lane);
    const uint4 p0 = shfl_u4(part, 0), p1 = shfl_u4(part, 1);
    const uint4 meta = shfl_u4(part, 2);  // k, req, njobs, gen
    const int16_t* A = (const int16_t*)(((unsigned long long)p0.y << 32) | p0.x);
    const int16_t* sv = (const int16_t*)(((unsigned long long)p0.w << 32) | p0.z);
    const int16_t* ev = (const int16_t*)(((unsigned long long)p1.y << 32) | p1.x);
    int16_t* out = (int16_t*)(((unsigned long long)p1.w << 32) | p1.z);
    fused_job<1>((int)meta.x, 1, A, sv, ev, out, rows, rowp, C, R, lane);
    if (lane == 0) {
      // outputs may be host memory: order them system-wide before counting
      __threadfence_system();
      const unsigned int done = atomicAdd(&req_ctr[meta.y], 1u) + 1u;
      if (done == meta.z) {
        // every job of the request has counted: reset the counter for the
        // slot's next request (admitted only after the host sees the flag)
        req_ctr[meta.y] = 0u;
        __threadfence_system();
        asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(&req_flag[meta.y]), "r"(meta.w)
                     : "memory");
      }
    }
    __syncwarp();
  }
}

cudaError_t launch_serve(const ServeJob* ring, uint32_t ring_mask, ServeCtl* ctl,
                         unsigned int* req_ctr, unsigned int* req_flag, unsigned long long idle_ns,
                         const DeviceInfo& info, cudaStream_t stream) {
  // (k_serve's shared-memory attribute is set per device by matvec_init_device)
  k_serve<<<(unsigned)info.num_sms, 32 * kServeWarps, kServeSmem, stream>>>(
      ring, ring_mask, ctl, req_ctr, req_flag, idle_ns);
  return cudaGetLastError();
}

static bool upload_fused_tables() {
  static Matrices M;
  static FwdFrags FF;
  static InvFrags IF;
  static std::once_flag once;
  std::call_once(once, [] {
    build_matrices(&M);
    build_fwd_frags(M, &FF);
    build_inv_frags(M, &IF);
  });
  return cudaMemcpyToSymbol(g_mv_fwd, &FF, sizeof(FF)) == cudaSuccess &&
         cudaMemcpyToSymbol(g_mv_inv, &IF, sizeof(IF)) == cudaSuccess &&
         cudaFuncSetAttribute(k_matvec_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kFusedSmem) == cudaSuccess &&
         cudaFuncSetAttribute(k_serve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kServeSmem) == cudaSuccess;
}

cudaError_t launch_matvec_fused(const FusedBatches& args, const DeviceInfo& info,
                                cudaStream_t stream) {
  FusedBatches a = args;  // group prefix: floor(8 / k) jobs per work item
  a.gfirst[0] = 0;
  for (int b = 0; b < a.nb; b++) {
    const int per = 8 / a.k[b], n = a.first[b + 1] - a.first[b];
    a.gfirst[b + 1] = a.gfirst[b] + (n + per - 1) / per;
  }
  const int total = a.gfirst[a.nb];
  if (total <= 0) return cudaSuccess;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_matvec_fused, 32 * kFusedWarps,
                                                kFusedSmem);
  long long blocks = (total + kFusedWarps - 1) / kFusedWarps;
  const long long cap = (long long)info.num_sms * (per_sm > 0 ? per_sm : 1);
  if (blocks > cap) blocks = cap;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(32 * kFusedWarps);
  cfg.dynamicSmemBytes = kFusedSmem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_matvec_fused, a);
}

bool matvec_init_device() { return upload_pair_constants() && upload_fused_tables(); }

template <int K>
static cudaError_t launch_basemul(const int16_t* A, int16_t* vec, int njobs, const DeviceInfo& info,
                                  cudaStream_t stream) {
  long long blocks = (njobs + 7) / 8;
  const long long cap = (long long)info.num_sms * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_basemul_acc<K>, A, vec, njobs);
}

cudaError_t launch_matvec(const MatvecPart* batches, int nb, const DeviceInfo& info,
                          cudaStream_t stream, int fwd_variant, int inv_variant,
                          long long chunk_vec_polys) {
  if (nb > kMaxSegs) return cudaErrorInvalidValue;
  // chunks of at most chunk_vec_polys vector polynomials, drawn from the
  // batches in order; a chunk holds at most one contiguous piece per batch
  size_t cur[kMaxSegs] = {0, 0, 0, 0};
  int b = 0;
  while (b < nb) {
    struct Piece {
      int b;
      size_t j0, nj;
    } pieces[kMaxSegs];
    int np = 0;
    long long room = chunk_vec_polys;
    while (b < nb && room > 0) {
      const MatvecPart& B = batches[b];
      if (cur[b] >= B.njobs) {
        b++;
        continue;
      }
      size_t take = (size_t)(room / B.k);
      if (take < 1) take = 1;
      if (take > B.njobs - cur[b]) take = B.njobs - cur[b];
      pieces[np++] = Piece{b, cur[b], take};
      cur[b] += take;
      room -= (long long)take * B.k;
      if (cur[b] >= B.njobs) b++;
    }
    if (np == 0) break;
    Seg fwd[kMaxSegs], inv[kMaxSegs];
    for (int p = 0; p < np; p++) {
      const MatvecPart& B = batches[pieces[p].b];
      const size_t v0 = pieces[p].j0 * (size_t)B.k * 256;
      const long long nvec = (long long)(pieces[p].nj * (size_t)B.k);
      fwd[p] = Seg{B.s + v0, B.out + v0, nvec, nullptr};
      inv[p] = Seg{B.out + v0, B.out + v0, nvec, B.e ? B.e + v0 : nullptr};
    }
    cudaError_t err = launch_mma_segs(false, fwd_variant, fwd, np, info, stream);
    for (int p = 0; p < np && err == cudaSuccess; p++) {
      const MatvecPart& B = batches[pieces[p].b];
      const size_t v0 = pieces[p].j0 * (size_t)B.k * 256;
      const size_t a0 = pieces[p].j0 * (size_t)B.k * (size_t)B.k * 256;
      const int nj = (int)pieces[p].nj;
      switch (B.k) {
        case 2: err = launch_basemul<2>(B.A + a0, B.out + v0, nj, info, stream); break;
        case 3: err = launch_basemul<3>(B.A + a0, B.out + v0, nj, info, stream); break;
        default: err = launch_basemul<4>(B.A + a0, B.out + v0, nj, info, stream); break;
      }
    }
    if (err == cudaSuccess) err = launch_mma_segs(true, inv_variant, inv, np, info, stream);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

}  // namespace tk
