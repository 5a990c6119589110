// tk_internal.h -- declarations shared between the kernel translation units and
// the C ABI layer (tk_api.cu).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tk {

struct DeviceInfo {
  int device = -1;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  int mma_ctas_per_sm[2] = {1, 1};  // [forward, inverse]
  size_t total_mem = 0;
};

// Uploads the constant fragment tables to the current device and fills the
// occupancy figures of the mma.sync kernels.
bool mma_init_device(DeviceInfo* info);

// Batched transform of npoly polynomials, src -> dst (src == dst for in place).
cudaError_t launch_mma(bool inverse, const int16_t* src, int16_t* dst, long long npoly,
                       const DeviceInfo& info, cudaStream_t stream);

// Kernel-side error flags (bounded waits that gave up), read and reset.
cudaError_t read_and_clear_status(unsigned* flags);

}  // namespace tk
