// tk_internal.h -- declarations shared between the kernel translation units and
// the C ABI layer (tk_api.cu).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tk {

// mma.sync kernel variants (CTA shape / pipeline depth):
//   0: 4 warps, 32-polynomial tiles, 3 slots   (4 CTAs/SM)
//   1: 8 warps, 64-polynomial tiles, 3 slots   (2 CTAs/SM)
//   2: 4 warps, 32-polynomial tiles, 2 slots   (6 CTAs/SM)
constexpr int kNumMmaVariants = 3;
// Largest batch one kernel launch covers (TMA coordinates are signed 32-bit).
constexpr long long kMaxLaunchPolys = 1ll << 30;

struct DeviceInfo {
  int device = -1;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  int mma_ctas_per_sm[2][kNumMmaVariants] = {{1, 1, 1}, {1, 1, 1}};  // [inverse][variant]
  size_t total_mem = 0;
};

// Uploads the constant fragment tables to the current device and fills the
// occupancy figures of the mma.sync kernels.
bool mma_init_device(DeviceInfo* info);

// Batched transform of npoly polynomials, src -> dst (src == dst for in place).
// Inverse only: a non-null addend (npoly polynomials) is added to the output
// with int16 wrap-around.
cudaError_t launch_mma(bool inverse, int variant, const int16_t* src, int16_t* dst,
                       long long npoly, const DeviceInfo& info, cudaStream_t stream,
                       const int16_t* addend = nullptr);

// CUresult of the calling thread's last tensor-map encode (launch_mma reports
// cudaErrorInvalidResourceHandle when an encode failed).
int last_encode_result();

// Matrix-vector jobs (tk_matvec.cu).  Chunks hold at most this many vector
// polynomials, so that intermediates stay in the 126 MB L2.
constexpr long long kMatvecChunkVecPolys = 131072;  // default (64 MiB); tk_set_option may change it
bool matvec_init_device();
cudaError_t launch_matvec(int k, size_t njobs, const int16_t* A, const int16_t* s,
                          const int16_t* e, int16_t* out, const DeviceInfo& info,
                          cudaStream_t stream, int fwd_variant, int inv_variant,
                          long long chunk_vec_polys);

// Kernel-side error flags (bounded waits that gave up), read and reset.
cudaError_t read_and_clear_status(unsigned* flags);

}  // namespace tk
