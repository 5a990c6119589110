// tk_matvec.cu -- batched ML-KEM matrix-vector jobs
//     out_i = invntt( sum_j basemul(A_ij, ntt(s_j)) ) + e_i,   i, j < k,
// the composition of the reference's ntt (ntt_bench/ref/ntt.c:80-95), basemul
// (ntt_bench/ref/ntt.c:139-146, applied pairwise as in ML-KEM's
// poly_basemul_montgomery) and invntt (ntt_bench/ref/ntt.c:106-126); the
// reference repository has no polyvec layer, so tko_matvec_job in the oracle
// restates the composition (barrett of the k-term sum before invntt, as ML-KEM's
// polyvec_basemul_acc_montgomery does).
//
// Execution, per uniform-k batch, in chunks of jobs whose vectors fit in L2:
//   1. forward NTT  s -> out           (k_ntt_mma, out of place)
//   2. basemul-acc  out <- A o out     (k_basemul_acc, in place per job)
//   3. inverse NTT  out -> out + e     (k_ntt_mma with addend)
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

namespace tk {

// Pair constants: pair t (coefficients 2t, 2t+1) of the NTT domain is the
// residue mod X^2 - z_t, z_t = +-17^brv7(64 + t/2) (sign + for even t); the
// reference's basemul multiplies by 2^-16 (Montgomery).  g_bm_zr[t] =
// z_t * 2^-16 mod q.
__device__ int32_t g_bm_zr[128];

constexpr uint32_t kRinv = 169;               // 2^-16 mod q
constexpr uint32_t kAccBias = 1073742318u;    // q * ceil(2^30 / q)

__device__ __forceinline__ uint32_t mulmod_lazy(uint32_t x, uint32_t c) {
  return red_lazy(x * c);  // x < q + 8, c < q: x * c < 2^24
}
// S in [0, 2^31): representative in [0, 3q).
__device__ __forceinline__ uint32_t red_wide(uint32_t s) {
  return s - __umulhi(s, 1290167u) * 3329u;
}

// One warp per job; lane l owns coefficient pairs 4l .. 4l+3 (16 bytes of every
// polynomial).  vec holds ntt(s) on entry and the accumulated products on
// exit; all k polynomials of a job are read before any is written.
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
    uint32_t B0[K][4], B1[K][4], Bz[K][4];
#pragma unroll
    for (int j = 0; j < K; j++) {
      const uint4 v = *(const uint4*)(vec + ((size_t)job * K + j) * 256 + 8 * lane);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t b0 = w[u] & 0xffffu, b1 = w[u] >> 16;  // forward output, [0, q)
        B0[j][u] = mulmod_lazy(b0, kRinv);
        B1[j][u] = mulmod_lazy(b1, kRinv);
        Bz[j][u] = mulmod_lazy(b1, zr[u]);
      }
    }
#pragma unroll
    for (int i = 0; i < K; i++) {
      int32_t acc0[4] = {0, 0, 0, 0}, acc1[4] = {0, 0, 0, 0};
#pragma unroll
      for (int j = 0; j < K; j++) {
        const uint4 v = __ldcs((const uint4*)(A + (((size_t)job * K + i) * K + j) * 256 + 8 * lane));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int32_t a0 = (int16_t)(w[u] & 0xffffu), a1 = (int32_t)w[u] >> 16;
          acc0[u] += a0 * (int32_t)B0[j][u] + a1 * (int32_t)Bz[j][u];
          acc1[u] += a0 * (int32_t)B1[j][u] + a1 * (int32_t)B0[j][u];
        }
      }
      // |acc| < 2K * 32768 * (q + 8) < 2^30: bias to non-negative, reduce.
      uint32_t o[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        o[u] = pack2(red_wide((uint32_t)acc0[u] + kAccBias), red_wide((uint32_t)acc1[u] + kAccBias));
      *(uint4*)(vec + ((size_t)job * K + i) * 256 + 8 * lane) = make_uint4(o[0], o[1], o[2], o[3]);
    }
  }
}

static bool upload_pair_constants() {
  // z_t = +-17^brv7(64 + t/2) mod q, times 2^-16
  int32_t zr[128];
  for (int t = 0; t < 128; t++) {
    unsigned k = 64 + t / 2, r = 0;
    for (int b = 0; b < 7; b++) r |= ((k >> b) & 1u) << (6 - b);
    int64_t z = 1;
    for (unsigned e = 0; e < r; e++) z = z * 17 % 3329;
    if (t & 1) z = (3329 - z) % 3329;
    zr[t] = (int32_t)(z * kRinv % 3329);
  }
  return cudaMemcpyToSymbol(g_bm_zr, zr, sizeof(zr)) == cudaSuccess;
}

bool matvec_init_device() { return upload_pair_constants(); }

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

cudaError_t launch_matvec(int k, size_t njobs, const int16_t* A, const int16_t* s,
                          const int16_t* e, int16_t* out, const DeviceInfo& info,
                          cudaStream_t stream, int fwd_variant, int inv_variant,
                          long long chunk_vec_polys) {
  size_t per_chunk = (size_t)chunk_vec_polys / (size_t)k;
  if (per_chunk < 1) per_chunk = 1;
  for (size_t j0 = 0; j0 < njobs; j0 += per_chunk) {
    const size_t nj = (njobs - j0) < per_chunk ? (njobs - j0) : per_chunk;
    const size_t v0 = j0 * (size_t)k * 256, a0 = j0 * (size_t)k * (size_t)k * 256;
    const long long nvec = (long long)(nj * (size_t)k);
    cudaError_t err = launch_mma(false, fwd_variant, s + v0, out + v0, nvec, info, stream);
    if (err != cudaSuccess) return err;
    switch (k) {
      case 2: err = launch_basemul<2>(A + a0, out + v0, (int)nj, info, stream); break;
      case 3: err = launch_basemul<3>(A + a0, out + v0, (int)nj, info, stream); break;
      default: err = launch_basemul<4>(A + a0, out + v0, (int)nj, info, stream); break;
    }
    if (err != cudaSuccess) return err;
    err = launch_mma(true, inv_variant, out + v0, out + v0, nvec, info, stream, e ? e + v0 : nullptr);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

}  // namespace tk
