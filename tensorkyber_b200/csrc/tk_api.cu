// tk_api.cu -- the C ABI (include/tk_ntt.h): argument checks, per-device set-up,
// dispatch to the sm_100a kernels, and the chunked host-memory path.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "../../include/tk_ntt.h"
#include "tk_host_sched.h"
#include "tk_internal.h"
#include "tk_tables.h"

namespace {

using tk::DeviceInfo;

constexpr int kMaxDevices = 64;

struct DeviceState {
  std::mutex mu;
  bool ready = false;
  DeviceInfo info;
  // host-path staging (allocated on the first host call for this device)
  std::mutex host_mu;
  int16_t* stage[3] = {nullptr, nullptr, nullptr};
  cudaStream_t streams[3] = {nullptr, nullptr, nullptr};
  size_t stage_polys = 0;
  // tk_matvec_host staging (grown on demand)
  std::mutex mv_mu;
  uint8_t* mv_stage = nullptr;
  size_t mv_bytes = 0;
  cudaStream_t mv_stream = nullptr;
};

DeviceState g_dev[kMaxDevices];
thread_local char t_err[256] = "";

// Kernel variant choice: forced by tk_set_variant (>= 0) or picked by size.
std::atomic<int> g_forced[2] = {{-1}, {-1}};
std::atomic<long long> g_matvec_chunk{tk::kMatvecChunkVecPolys};
// Host path: polynomials per chunk (TK_OPT_HOST_CHUNK_POLYS), at most the
// staging buffers' kHostStagePolys.
constexpr size_t kHostStagePolys = (size_t)1 << 15;  // 16 MiB per staging buffer
constexpr long long kHostChunkDefault = 1 << 15;
std::atomic<long long> g_host_chunk{kHostChunkDefault};
std::atomic<int> g_matvec_mode{TK_MATVEC_TILED};

const char* const kVariantNames[tk::kNumMmaVariants] = {
    "mma.sync 4 warps x 32-poly tiles, 3-slot TMA ring",
    "mma.sync 8 warps x 64-poly tiles, 3-slot TMA ring",
    "mma.sync 4 warps x 32-poly tiles, 2-slot TMA ring",
    "mma.sync 4 warps x 32-poly tiles, 2-slot TMA ring, int32 stage-1 tile",
    "tcgen05 kind::i8, 128-poly tiles, TMEM accumulators and second-stage operand",
};

// Autotuned choice per direction and size bucket floor(log2(npoly)); -1 =
// not tuned: variant 3 for the forward; for the inverse variant 0 below 2^19
// polynomials and variant 2 from there (the fastest shapes measured at 2^18
// and 2^20).
constexpr int kBuckets = 33;
std::atomic<int> g_tuned[2][kBuckets];
struct TunedInit {
  TunedInit() {
    for (auto& d : g_tuned)
      for (auto& b : d) b.store(-1);
  }
} g_tuned_init;

int size_bucket(size_t npoly) {
  int b = 0;
  while (b + 1 < kBuckets && ((size_t)1 << (b + 1)) <= npoly) b++;
  return b;
}

int choose_variant(bool inverse, size_t npoly) {
  const int f = g_forced[inverse ? 1 : 0].load(std::memory_order_relaxed);
  if (f >= 0) return f;
  const int t = g_tuned[inverse ? 1 : 0][size_bucket(npoly)].load(std::memory_order_relaxed);
  if (t >= 0) return t;
  // untuned: the measured best per direction (forward: the int32-tile
  // mma.sync kernel everywhere; inverse: the tcgen05 kernel from 2^18
  // polynomials, where it leads, the 3-slot mma.sync kernel below, where the
  // tcgen05 kernel's larger CTA costs more to start)
  return inverse ? (npoly >= ((size_t)1 << 18) ? tk::kTc5Variant : 0) : 3;
}

void set_err(const char* what, cudaError_t e) {
  snprintf(t_err, sizeof(t_err), "%s: %s", what, cudaGetErrorString(e));
}
void set_msg(const char* msg) { snprintf(t_err, sizeof(t_err), "%s", msg); }

// Current device of the calling thread.  The first call on a thread also
// binds the device's primary context to the thread (cudaSetDevice), because
// the tensor-map encoder is a driver call that needs a current context even
// when the thread has made no runtime call yet.
thread_local int t_bound_device = -1;

int current_device(int* dev) {
  cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) {
    set_err("cudaGetDevice", e);
    return TK_ERR_NO_DEVICE;
  }
  if (*dev < 0 || *dev >= kMaxDevices) {
    set_msg("device ordinal out of range");
    return TK_ERR_NO_DEVICE;
  }
  if (t_bound_device != *dev) {
    if ((e = cudaSetDevice(*dev)) != cudaSuccess) {
      set_err("cudaSetDevice", e);
      return TK_ERR_NO_DEVICE;
    }
    t_bound_device = *dev;
  }
  return TK_SUCCESS;
}

void set_launch_err(cudaError_t e) {
  if (e == cudaErrorInvalidResourceHandle)
    snprintf(t_err, sizeof(t_err), "cuTensorMapEncodeTiled failed (CUresult %d)",
             tk::last_encode_result());
  else
    set_err("kernel launch", e);
}

// Set-up of the current device; idempotent and thread-safe.
int ensure_ready(int dev, DeviceInfo** out) {
  DeviceState& S = g_dev[dev];
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.ready) {
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, dev);
    if (e != cudaSuccess) {
      set_err("cudaGetDeviceProperties", e);
      return TK_ERR_NO_DEVICE;
    }
    if (p.major != 10 || p.minor != 0) {
      snprintf(t_err, sizeof(t_err), "device %d is sm_%d%d; this build targets sm_100a only", dev,
               p.major, p.minor);
      return TK_ERR_NO_DEVICE;
    }
    S.info.device = dev;
    S.info.num_sms = p.multiProcessorCount;
    S.info.cc_major = p.major;
    S.info.cc_minor = p.minor;
    S.info.total_mem = p.totalGlobalMem;
    if (!tk::mma_init_device(&S.info) || !tk::matvec_init_device() ||
        !tk::tc5_init_device(&S.info)) {
      set_err("kernel set-up", cudaGetLastError());
      return TK_ERR_CUDA;
    }
    S.ready = true;
  }
  *out = &S.info;
  return TK_SUCCESS;
}

int check_device_ptr(const void* p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_err("cudaPointerGetAttributes", e);
    return TK_ERR_NOT_DEVICE_MEMORY;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return TK_SUCCESS;
  if (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr && a.devicePointer == p)
    return TK_SUCCESS;  // mapped pinned memory with identical addresses
  set_msg("pointer is not device-accessible memory");
  return TK_ERR_NOT_DEVICE_MEMORY;
}

int run_device(bool inverse, const int16_t* in, int16_t* out, size_t npoly, cudaStream_t st) {
  t_err[0] = 0;
  if (npoly == 0) return TK_SUCCESS;
  if (!in || !out) {
    set_msg("NULL polynomial pointer");
    return TK_ERR_INVALID_VALUE;
  }
  if (npoly > TK_MAX_POLYS) {
    set_msg("npoly above TK_MAX_POLYS");
    return TK_ERR_TOO_LARGE;
  }
  if (((uintptr_t)in & 15u) || ((uintptr_t)out & 15u)) {
    set_msg("polynomial buffers must be 16-byte aligned");
    return TK_ERR_MISALIGNED;
  }
  const uintptr_t bytes = (uintptr_t)npoly * 512u;
  if (in != out) {
    const uintptr_t a = (uintptr_t)in, b = (uintptr_t)out;
    if (a < b + bytes && b < a + bytes) {
      set_msg("input and output overlap without being identical");
      return TK_ERR_INVALID_VALUE;
    }
  }
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  DeviceInfo* info;
  rc = ensure_ready(dev, &info);
  if (rc) return rc;
  rc = check_device_ptr(in);
  if (rc) return rc;
  if (in != out && (rc = check_device_ptr(out))) return rc;
  cudaError_t e = tk::launch_mma(inverse, choose_variant(inverse, npoly), in, out,
                                 (long long)npoly, *info, st);
  if (e != cudaSuccess) {
    set_launch_err(e);
    return TK_ERR_CUDA;
  }
  return TK_SUCCESS;
}

// Host path: chunks of at most stage_polys polynomials (sized by
// tk::host_chunk_size) rotate through kHostStages device buffers and streams,
// so the H2D copy of chunk c+1, the kernel of chunk c and the D2H copy of
// chunk c-1 overlap, and an upload waits only for the download kHostStages
// chunks back.
constexpr int kHostStages = 3;  // 4 measured the same
using tk::host_chunk_size;
int run_host(bool inverse, int16_t* polys, size_t npoly) {
  t_err[0] = 0;
  if (npoly == 0) return TK_SUCCESS;
  if (!polys) {
    set_msg("NULL polynomial pointer");
    return TK_ERR_INVALID_VALUE;
  }
  if (npoly > TK_MAX_POLYS) {
    set_msg("npoly above TK_MAX_POLYS");
    return TK_ERR_TOO_LARGE;
  }
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  DeviceInfo* info;
  rc = ensure_ready(dev, &info);
  if (rc) return rc;
  DeviceState& S = g_dev[dev];
  std::lock_guard<std::mutex> lk(S.host_mu);
  cudaError_t e;
  if (!S.stage[0]) {
    S.stage_polys = kHostStagePolys;
    for (int i = 0; i < kHostStages; i++) {
      if ((e = cudaMalloc(&S.stage[i], S.stage_polys * 512u)) != cudaSuccess ||
          (e = cudaStreamCreateWithFlags(&S.streams[i], cudaStreamNonBlocking)) != cudaSuccess) {
        set_err("host-path staging set-up", e);
        for (int j = 0; j < kHostStages; j++) {
          if (S.stage[j]) cudaFree(S.stage[j]);
          if (S.streams[j]) cudaStreamDestroy(S.streams[j]);
          S.stage[j] = nullptr;
          S.streams[j] = nullptr;
        }
        return TK_ERR_CUDA;
      }
    }
  }
  size_t chunk = (size_t)g_host_chunk.load(std::memory_order_relaxed);
  if (chunk > S.stage_polys) chunk = S.stage_polys;
  size_t done = 0;
  int c = 0;
  e = cudaSuccess;
  while (done < npoly && e == cudaSuccess) {
    const size_t n = host_chunk_size(c, npoly - done, chunk);
    cudaStream_t st = S.streams[c % kHostStages];
    int16_t* buf = S.stage[c % kHostStages];
    e = cudaMemcpyAsync(buf, polys + done * 256, n * 512u, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = tk::launch_mma(inverse, choose_variant(inverse, n), buf, buf, (long long)n, *info, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(polys + done * 256, buf, n * 512u, cudaMemcpyDeviceToHost, st);
    done += n;
    c++;
  }
  for (int i = 0; i < kHostStages; i++) {
    cudaError_t e2 = cudaStreamSynchronize(S.streams[i]);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) {
    set_err("host-path transform", e);
    return TK_ERR_CUDA;
  }
  return TK_SUCCESS;
}

}  // namespace

namespace tk {
bool host_span_one_copy(const void* p, size_t bytes) {
  static PFN_cuPointerGetAttribute_v4000 get_attr = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    return cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) ==
                       cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? (PFN_cuPointerGetAttribute_v4000)f
               : nullptr;
  }();
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeUnregistered) return true;
  if (a.type != cudaMemoryTypeHost || !get_attr) return false;
  // page-locked: the span must stay inside the allocation
  CUdeviceptr start = 0;
  size_t size = 0;
  const CUdeviceptr dp = (CUdeviceptr)(a.devicePointer ? a.devicePointer : p);
  if (get_attr(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, dp) != CUDA_SUCCESS ||
      get_attr(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, dp) != CUDA_SUCCESS)
    return false;
  return dp >= start && dp + bytes <= start + size;
}

int api_device_info(int device, DeviceInfo** info) {
  if (device < 0 || device >= kMaxDevices) return TK_ERR_INVALID_VALUE;
  return ensure_ready(device, info);
}
}  // namespace tk

extern "C" {

int tk_ntt(int16_t* polys, size_t npoly, tk_stream_t stream) {
  return run_device(false, polys, polys, npoly, (cudaStream_t)stream);
}
int tk_invntt(int16_t* polys, size_t npoly, tk_stream_t stream) {
  return run_device(true, polys, polys, npoly, (cudaStream_t)stream);
}
int tk_ntt_oop(const int16_t* in, int16_t* out, size_t npoly, tk_stream_t stream) {
  return run_device(false, in, out, npoly, (cudaStream_t)stream);
}
int tk_invntt_oop(const int16_t* in, int16_t* out, size_t npoly, tk_stream_t stream) {
  return run_device(true, in, out, npoly, (cudaStream_t)stream);
}
int tk_ntt_host(int16_t* polys, size_t npoly) { return run_host(false, polys, npoly); }

// Forward transform of an input form (1: small int16, 2/3: packed) on device
// buffers; in_bytes per polynomial of the input.
static int run_form(int form, const void* in, int16_t* out, size_t npoly, size_t in_bytes,
                    cudaStream_t st) {
  t_err[0] = 0;
  if (npoly == 0) return TK_SUCCESS;
  if (!in || !out) {
    set_msg("NULL buffer pointer");
    return TK_ERR_INVALID_VALUE;
  }
  if (npoly > TK_MAX_POLYS) {
    set_msg("npoly above TK_MAX_POLYS");
    return TK_ERR_TOO_LARGE;
  }
  if (((uintptr_t)in & 15u) || ((uintptr_t)out & 15u)) {
    set_msg("buffers must be 16-byte aligned");
    return TK_ERR_MISALIGNED;
  }
  const uintptr_t a = (uintptr_t)in, b = (uintptr_t)out;
  const uintptr_t na = (uintptr_t)npoly * in_bytes, nb = (uintptr_t)npoly * 512u;
  const bool same = form == 1 && a == b;
  if (!same && a < b + nb && b < a + na) {
    set_msg(form == 1 ? "input and output overlap without being identical"
                      : "packed input overlaps the output");
    return TK_ERR_INVALID_VALUE;
  }
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  DeviceInfo* info;
  if ((rc = ensure_ready(dev, &info))) return rc;
  if ((rc = check_device_ptr(in))) return rc;
  if (!same && (rc = check_device_ptr(out))) return rc;
  const cudaError_t e = tk::launch_fwd_form(form, in, out, (long long)npoly, *info, st);
  if (e != cudaSuccess) {
    set_launch_err(e);
    return TK_ERR_CUDA;
  }
  return TK_SUCCESS;
}

int tk_ntt_small(const int16_t* in, int16_t* out, size_t npoly, tk_stream_t stream) {
  return run_form(1, in, out, npoly, 512, (cudaStream_t)stream);
}

int tk_ntt_packed(const void* packed, int bits, int16_t* out, size_t npoly, tk_stream_t stream) {
  if (bits != 2 && bits != 3) {
    t_err[0] = 0;
    set_msg("tk_ntt_packed: bits must be 2 or 3");
    return TK_ERR_INVALID_VALUE;
  }
  return run_form(bits, packed, out, npoly, bits == 2 ? 64 : 128, (cudaStream_t)stream);
}

// Host-side packing (the format of tk_ntt_packed); a plain data conversion,
// not a transform.
int tk_pack_small(const int16_t* polys, size_t npoly, int bits, void* packed) {
  t_err[0] = 0;
  if (bits != 2 && bits != 3) {
    set_msg("tk_pack_small: bits must be 2 or 3");
    return TK_ERR_INVALID_VALUE;
  }
  if (npoly == 0) return TK_SUCCESS;
  if (!polys || !packed) {
    set_msg("tk_pack_small: NULL pointer");
    return TK_ERR_INVALID_VALUE;
  }
  const int per = 8 / bits, lo = -(1 << (bits - 1)), hi = (1 << (bits - 1)) - 1;
  const size_t row = 256 / per;
  uint8_t* dst = (uint8_t*)packed;
  for (size_t p = 0; p < npoly; p++) {
    const int16_t* x = polys + p * 256;
    uint8_t* d = dst + p * row;
    memset(d, 0, row);
    for (int i = 0; i < 256; i++) {
      if (x[i] < lo || x[i] > hi) {
        snprintf(t_err, sizeof(t_err),
                 "tk_pack_small: polynomial %zu coefficient %d = %d outside [%d, %d]", p, i,
                 (int)x[i], lo, hi);
        return TK_ERR_INVALID_VALUE;
      }
      d[i / per] |= (uint8_t)((x[i] & ((1 << bits) - 1)) << ((i % per) * bits));
    }
  }
  return TK_SUCCESS;
}

static bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + nb && y < x + na;
}

// Checks of a batch list common to the device and host forms; *nonempty =
// batches with work.  host: pointers are host memory (no alignment or overlap
// rule, the data is staged).
static int validate_matvec(const tk_matvec_batch* batches, int nbatches, bool host,
                           int* nonempty_out) {
  if (nbatches < 0 || (nbatches > 0 && !batches)) {
    set_msg("tk_matvec: bad batch list");
    return TK_ERR_INVALID_VALUE;
  }
  int nonempty = 0;
  for (int b = 0; b < nbatches; b++) {  // validate everything before launching anything
    const tk_matvec_batch& B = batches[b];
    if (B.njobs == 0) continue;
    nonempty++;
    if (B.k < 2 || B.k > 4) {
      set_msg("tk_matvec: k must be 2, 3 or 4");
      return TK_ERR_INVALID_VALUE;
    }
    if (!B.A || !B.s || !B.out) {
      set_msg("tk_matvec: NULL A, s or out");
      return TK_ERR_INVALID_VALUE;
    }
    if (B.njobs > ((size_t)1 << 28)) {
      set_msg("tk_matvec: too many jobs in one batch");
      return TK_ERR_TOO_LARGE;
    }
    if (host) continue;
    if ((((uintptr_t)B.A | (uintptr_t)B.s | (uintptr_t)B.e | (uintptr_t)B.out) & 15u) != 0) {
      set_msg("tk_matvec: buffers must be 16-byte aligned");
      return TK_ERR_MISALIGNED;
    }
    const size_t vb = B.njobs * (size_t)B.k * 512u, ab = vb * (size_t)B.k;
    if (overlaps(B.out, vb, B.A, ab) || (B.e && overlaps(B.out, vb, B.e, vb)) ||
        (B.s != B.out && overlaps(B.out, vb, B.s, vb))) {
      set_msg("tk_matvec: out overlaps A or e, or partially overlaps s");
      return TK_ERR_INVALID_VALUE;
    }
  }
  *nonempty_out = nonempty;
  return TK_SUCCESS;
}

// Launches a validated batch list of device buffers.
static int launch_matvec_batches(const tk_matvec_batch* batches, int nbatches,
                                 const DeviceInfo* info, cudaStream_t stream) {
  const int mode = g_matvec_mode.load(std::memory_order_relaxed);
  if (mode == TK_MATVEC_TILED) {  // one tile-kernel launch per kMaxSegs batches
    tk::MatvecPart parts[tk::kMaxSegs];
    int np = 0;
    for (int b = 0; b <= nbatches; b++) {
      if (b < nbatches && batches[b].njobs != 0) {
        const tk_matvec_batch& B = batches[b];
        parts[np++] = tk::MatvecPart{B.k, B.njobs, B.A, B.s, B.e, B.out};
      }
      if (np == tk::kMaxSegs || (b == nbatches && np > 0)) {
        cudaError_t e = tk::launch_matvec_tile(parts, np, *info, stream);
        if (e != cudaSuccess) {
          set_launch_err(e);
          return TK_ERR_CUDA;
        }
        np = 0;
      }
    }
    return TK_SUCCESS;
  }
  if (mode == TK_MATVEC_FUSED) {
    // single-launch fused kernel, up to three batches per launch
    tk::FusedBatches fb{};
    int b = 0;
    while (b < nbatches) {
      fb.nb = 0;
      fb.first[0] = 0;
      for (; b < nbatches && fb.nb < 3; b++) {
        const tk_matvec_batch& B = batches[b];
        if (B.njobs == 0) continue;
        fb.k[fb.nb] = B.k;
        fb.A[fb.nb] = B.A;
        fb.s[fb.nb] = B.s;
        fb.e[fb.nb] = B.e;
        fb.out[fb.nb] = B.out;
        fb.first[fb.nb + 1] = fb.first[fb.nb] + (int)B.njobs;
        fb.nb++;
      }
      if (fb.nb == 0) break;
      cudaError_t e = tk::launch_matvec_fused(fb, *info, (cudaStream_t)stream);
      if (e != cudaSuccess) {
        set_launch_err(e);
        return TK_ERR_CUDA;
      }
    }
    return TK_SUCCESS;
  }
  // non-empty batches, up to kMaxSegs per pipeline call (they share its NTT launches)
  const long long chunk = g_matvec_chunk.load(std::memory_order_relaxed);
  tk::MatvecPart parts[tk::kMaxSegs];
  int np = 0;
  for (int b = 0; b <= nbatches; b++) {
    if (b < nbatches && batches[b].njobs != 0) {
      const tk_matvec_batch& B = batches[b];
      parts[np++] = tk::MatvecPart{B.k, B.njobs, B.A, B.s, B.e, B.out};
    }
    if (np == tk::kMaxSegs || (b == nbatches && np > 0)) {
      cudaError_t e = tk::launch_matvec(parts, np, *info, stream,
                                        choose_variant(false, (size_t)chunk),
                                        choose_variant(true, (size_t)chunk), chunk);
      if (e != cudaSuccess) {
        set_launch_err(e);
        return TK_ERR_CUDA;
      }
      np = 0;
    }
  }
  return TK_SUCCESS;
}

int tk_matvec(const tk_matvec_batch* batches, int nbatches, tk_stream_t stream) {
  t_err[0] = 0;
  int nonempty = 0;
  int rc = validate_matvec(batches, nbatches, false, &nonempty);
  if (rc || nonempty == 0) return rc;
  int dev;
  if ((rc = current_device(&dev))) return rc;
  DeviceInfo* info;
  if ((rc = ensure_ready(dev, &info))) return rc;
  for (int b = 0; b < nbatches; b++) {
    const tk_matvec_batch& B = batches[b];
    if (B.njobs == 0) continue;
    const void* ptrs[4] = {B.A, B.s, B.out, B.e};
    for (const void* p : ptrs)
      if (p && (rc = check_device_ptr(p))) return rc;
  }
  return launch_matvec_batches(batches, nbatches, info, (cudaStream_t)stream);
}

int tk_matvec_host(const tk_matvec_batch* batches, int nbatches) {
  t_err[0] = 0;
  int nonempty = 0;
  int rc = validate_matvec(batches, nbatches, true, &nonempty);
  if (rc || nonempty == 0) return rc;
  constexpr size_t kAlign = 256, kMaxStage = (size_t)8 << 30;
  auto up = [](size_t n) { return (n + kAlign - 1) & ~(kAlign - 1); };
  size_t need = 0;
  for (int b = 0; b < nbatches; b++) {
    const tk_matvec_batch& B = batches[b];
    const size_t vb = B.njobs * (size_t)B.k * 512u;
    need += up(vb * (size_t)B.k + vb * (B.e ? 3 : 2));
  }
  if (need > kMaxStage) {
    set_msg("tk_matvec_host: batch list above the 8 GiB staging limit");
    return TK_ERR_TOO_LARGE;
  }
  int dev;
  if ((rc = current_device(&dev))) return rc;
  DeviceInfo* info;
  if ((rc = ensure_ready(dev, &info))) return rc;
  DeviceState& S = g_dev[dev];
  std::lock_guard<std::mutex> lk(S.mv_mu);
  cudaError_t e = cudaSuccess;
  if (!S.mv_stream) e = cudaStreamCreateWithFlags(&S.mv_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess && S.mv_bytes < need) {
    if (S.mv_stage) cudaFree(S.mv_stage);
    S.mv_stage = nullptr;
    S.mv_bytes = 0;
    e = cudaMalloc(&S.mv_stage, need);
    if (e == cudaSuccess) S.mv_bytes = need;
  }
  if (e != cudaSuccess) {
    set_err("tk_matvec_host staging", e);
    return e == cudaErrorMemoryAllocation ? TK_ERR_TOO_LARGE : TK_ERR_CUDA;
  }
  std::vector<tk_matvec_batch> dev_batches((size_t)nbatches);
  cudaStream_t st = S.mv_stream;
  size_t off = 0;
  for (int b = 0; b < nbatches && e == cudaSuccess; b++) {
    const tk_matvec_batch& B = batches[b];
    tk_matvec_batch& D = dev_batches[(size_t)b];
    D = B;
    if (B.njobs == 0) continue;
    // staging block A | s | e | out, unpadded (whole 512-byte polynomials), so
    // inputs the caller keeps contiguous arrive in one copy
    const size_t vb = B.njobs * (size_t)B.k * 512u, ab = vb * (size_t)B.k;
    int16_t* dA = (int16_t*)(S.mv_stage + off);
    int16_t* ds = (int16_t*)(S.mv_stage + off + ab);
    int16_t* de = B.e ? (int16_t*)(S.mv_stage + off + ab + vb) : nullptr;
    int16_t* dout = (int16_t*)(S.mv_stage + off + ab + vb * (B.e ? 2 : 1));
    off += up(ab + vb * (B.e ? 3 : 2));
    const bool packed = (const uint8_t*)B.s == (const uint8_t*)B.A + ab &&
                        (!B.e || (const uint8_t*)B.e == (const uint8_t*)B.s + vb) &&
                        tk::host_span_one_copy(B.A, ab + vb * (B.e ? 2 : 1));
    if (packed) {
      e = cudaMemcpyAsync(dA, B.A, ab + vb * (B.e ? 2 : 1), cudaMemcpyHostToDevice, st);
    } else {
      e = cudaMemcpyAsync(dA, B.A, ab, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(ds, B.s, vb, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess && de) e = cudaMemcpyAsync(de, B.e, vb, cudaMemcpyHostToDevice, st);
    }
    D.A = dA;
    D.s = ds;
    D.e = de;
    D.out = dout;
  }
  if (e == cudaSuccess) {
    rc = launch_matvec_batches(dev_batches.data(), nbatches, info, st);
    if (rc) {
      cudaStreamSynchronize(st);
      return rc;
    }
  }
  for (int b = 0; b < nbatches && e == cudaSuccess; b++) {
    const tk_matvec_batch& B = batches[b];
    if (B.njobs == 0) continue;
    e = cudaMemcpyAsync(B.out, dev_batches[(size_t)b].out, B.njobs * (size_t)B.k * 512u,
                        cudaMemcpyDeviceToHost, st);
  }
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) {
    set_err("tk_matvec_host", e);
    return TK_ERR_CUDA;
  }
  return TK_SUCCESS;
}

// ---- tk_matvec_host_noalloc: staging in a static device array ----------------
// The same copy-in / kernels / copy-out sequence as tk_matvec_host, but the
// staging block is a file-scope device array of TK_NOALLOC_SCRATCH_BYTES
// (allocated with the module, never by a call) and the work runs on the
// caller's stream: no cudaMalloc, cudaFree or stream creation on any call.
// Per device, the first call (with that device current) looks up the array's
// address with cudaGetSymbolAddress.  Every scratch byte the kernels read is
// written earlier in the same call (inputs copied in; outputs written by the
// kernels before they are copied out), so nothing has to start at zero.  One
// array per device: calls that overlap in time on one device race.
static __device__ __align__(256) uint8_t g_noalloc_scratch[TK_NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[kMaxDevices];

constexpr int kNoallocMaxBatches = 16;

int tk_matvec_host_noalloc(const tk_matvec_batch* batches, int nbatches, tk_stream_t stream) {
  t_err[0] = 0;
  int nonempty = 0;
  int rc = validate_matvec(batches, nbatches, true, &nonempty);
  if (rc || nonempty == 0) return rc;
  if (nbatches > kNoallocMaxBatches) {  // before any device work
    set_msg("tk_matvec_host_noalloc: at most 16 batches per call");
    return TK_ERR_INVALID_VALUE;
  }
  size_t need = 0;
  for (int b = 0; b < nbatches; b++) {
    const tk_matvec_batch& B = batches[b];
    const size_t vb = B.njobs * (size_t)B.k * 512u;
    need += (vb * (size_t)B.k + vb * (B.e ? 3 : 2) + 255) & ~(size_t)255;
  }
  if (need > TK_NOALLOC_SCRATCH_BYTES) {
    snprintf(t_err, sizeof(t_err),
             "tk_matvec_host_noalloc: the batch list needs %zu bytes of staging, above the "
             "%d-byte static scratch",
             need, TK_NOALLOC_SCRATCH_BYTES);
    return TK_ERR_TOO_LARGE;
  }
  int dev;
  if ((rc = current_device(&dev))) return rc;
  DeviceInfo* info;
  if ((rc = ensure_ready(dev, &info))) return rc;
  uint8_t* scratch;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_err("tk_matvec_host_noalloc: cudaGetSymbolAddress of the static scratch", e);
        return TK_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = p;
    }
    scratch = (uint8_t*)g_noalloc_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  tk_matvec_batch dev_batches[kNoallocMaxBatches] = {};
  cudaError_t e = cudaSuccess;
  size_t off = 0;
  for (int b = 0; b < nbatches && e == cudaSuccess; b++) {
    const tk_matvec_batch& B = batches[b];
    tk_matvec_batch& D = dev_batches[b];
    D = B;
    if (B.njobs == 0) continue;
    const size_t vb = B.njobs * (size_t)B.k * 512u, ab = vb * (size_t)B.k;
    int16_t* dA = (int16_t*)(scratch + off);
    int16_t* ds = (int16_t*)(scratch + off + ab);
    int16_t* de = B.e ? (int16_t*)(scratch + off + ab + vb) : nullptr;
    int16_t* dout = (int16_t*)(scratch + off + ab + vb * (B.e ? 2 : 1));
    off += (ab + vb * (B.e ? 3 : 2) + 255) & ~(size_t)255;
    e = cudaMemcpyAsync(dA, B.A, ab, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, B.s, vb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && de) e = cudaMemcpyAsync(de, B.e, vb, cudaMemcpyHostToDevice, st);
    D.A = dA;
    D.s = ds;
    D.e = de;
    D.out = dout;
  }
  if (e == cudaSuccess) {
    rc = launch_matvec_batches(dev_batches, nbatches, info, st);
    if (rc) {
      cudaStreamSynchronize(st);
      return rc;
    }
  }
  for (int b = 0; b < nbatches && e == cudaSuccess; b++) {
    const tk_matvec_batch& B = batches[b];
    if (B.njobs == 0) continue;
    e = cudaMemcpyAsync(B.out, dev_batches[b].out, B.njobs * (size_t)B.k * 512u,
                        cudaMemcpyDeviceToHost, st);
  }
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) {
    set_err("tk_matvec_host_noalloc", e);
    return TK_ERR_CUDA;
  }
  return TK_SUCCESS;
}

int tk_invntt_host(int16_t* polys, size_t npoly) { return run_host(true, polys, npoly); }

int tk_init(int device) {
  t_err[0] = 0;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_err("cudaGetDeviceCount", e);
    return TK_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n || device >= kMaxDevices) {
    set_msg("device ordinal out of range");
    return TK_ERR_INVALID_VALUE;
  }
  int prev;
  if ((e = cudaGetDevice(&prev)) != cudaSuccess) {
    set_err("cudaGetDevice", e);
    return TK_ERR_NO_DEVICE;
  }
  if ((e = cudaSetDevice(device)) != cudaSuccess) {
    set_err("cudaSetDevice", e);
    return TK_ERR_NO_DEVICE;
  }
  DeviceInfo* info;
  int rc = ensure_ready(device, &info);
  cudaSetDevice(prev);
  return rc;
}

int tk_selftest_bounded_wait(int device, double seconds) {
  t_err[0] = 0;
  if (!(seconds > 0.0) || seconds > 10.0) {
    set_msg("tk_selftest_bounded_wait: seconds must be in (0, 10]");
    return TK_ERR_INVALID_VALUE;
  }
  int rc = tk_init(device);
  if (rc) return rc;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaError_t e = tk::launch_selftest_wait((unsigned long long)(seconds * 1e9), 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_err("tk_selftest_bounded_wait", e);
    return TK_ERR_CUDA;
  }
  return TK_SUCCESS;
}

int tk_device_status(int device, unsigned* flags) {
  t_err[0] = 0;
  if (!flags) return TK_ERR_INVALID_VALUE;
  int rc = tk_init(device);
  if (rc) return rc;
  int prev;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = tk::read_and_clear_status(flags);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_err("tk_device_status", e);
    return TK_ERR_CUDA;
  }
  return *flags ? TK_ERR_KERNEL_TIMEOUT : TK_SUCCESS;
}

const char* tk_status_string(int status) {
  switch (status) {
    case TK_SUCCESS: return "success";
    case TK_ERR_INVALID_VALUE: return "invalid value";
    case TK_ERR_MISALIGNED: return "misaligned polynomial buffer";
    case TK_ERR_TOO_LARGE: return "batch too large";
    case TK_ERR_NO_DEVICE: return "no usable sm_100 device";
    case TK_ERR_CUDA: return "CUDA runtime error";
    case TK_ERR_NOT_DEVICE_MEMORY: return "pointer is not device memory";
    case TK_ERR_KERNEL_TIMEOUT: return "kernel bounded wait timed out";
    case TK_ERR_TIMEOUT: return "host wait timed out";
    default: return "unknown status";
  }
}

const char* tk_last_error(void) { return t_err; }

int tk_variant_count(void) { return tk::kNumMmaVariants; }

const char* tk_variant_name(int variant) {
  if (variant < 0 || variant >= tk::kNumMmaVariants) return "";
  return kVariantNames[variant];
}

int tk_set_variant(int direction, int variant) {
  t_err[0] = 0;
  if ((direction != TK_FORWARD && direction != TK_INVERSE) ||
      (variant != -1 && !tk::variant_valid(direction == TK_INVERSE, variant))) {
    set_msg("tk_set_variant: bad direction or variant");
    return TK_ERR_INVALID_VALUE;
  }
  g_forced[direction == TK_INVERSE ? 1 : 0].store(variant);
  return TK_SUCCESS;
}

int tk_set_option(int option, long long value) {
  t_err[0] = 0;
  switch (option) {
    case TK_OPT_MATVEC_CHUNK_POLYS:
      if (value < 0 || value > (1ll << 30)) break;
      g_matvec_chunk.store(value == 0 ? tk::kMatvecChunkVecPolys : value);
      return TK_SUCCESS;
    case TK_OPT_MATVEC_MODE:
      if (value != TK_MATVEC_PIPELINE && value != TK_MATVEC_FUSED && value != TK_MATVEC_TILED)
        break;
      g_matvec_mode.store((int)value);
      return TK_SUCCESS;
    case TK_OPT_HOST_CHUNK_POLYS:
      if (value < 0 || value > (long long)kHostStagePolys) break;
      g_host_chunk.store(value == 0 ? kHostChunkDefault : value);
      return TK_SUCCESS;
    default:
      break;
  }
  set_msg("tk_set_option: unknown option or value out of range");
  return TK_ERR_INVALID_VALUE;
}

long long tk_get_option(int option) {
  switch (option) {
    case TK_OPT_MATVEC_CHUNK_POLYS: return g_matvec_chunk.load();
    case TK_OPT_MATVEC_MODE: return g_matvec_mode.load();
    case TK_OPT_HOST_CHUNK_POLYS: return g_host_chunk.load();
    default: return -TK_ERR_INVALID_VALUE;
  }
}

int tk_get_variant(int direction, size_t npoly) {
  if (direction != TK_FORWARD && direction != TK_INVERSE) return -TK_ERR_INVALID_VALUE;
  return choose_variant(direction == TK_INVERSE, npoly);
}
int tk_abi_version(void) { return TK_ABI_VERSION; }

// ---- autotuner ----------------------------------------------------------------
static int load_tuning(const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return TK_ERR_INVALID_VALUE;
  char head[64] = {0};
  int rc = TK_ERR_INVALID_VALUE;
  if (fgets(head, sizeof(head), f) && strncmp(head, "tk-autotune 1", 13) == 0) {
    int dir, bucket, variant;
    double us;
    int n = 0;
    while (fscanf(f, "%d %d %d %lf", &dir, &bucket, &variant, &us) == 4) {
      if (dir < 0 || dir > 1 || bucket < 0 || bucket >= kBuckets ||
          !tk::variant_valid(dir == 1, variant)) {
        n = -1;
        break;
      }
      g_tuned[dir][bucket].store(variant);
      n++;
    }
    rc = n > 0 ? TK_SUCCESS : TK_ERR_INVALID_VALUE;
  }
  fclose(f);
  return rc;
}

int tk_autotune(int device, size_t max_npoly, const char* cache_path) {
  t_err[0] = 0;
  if (cache_path && load_tuning(cache_path) == TK_SUCCESS) return TK_SUCCESS;
  if (max_npoly == 0 || max_npoly > TK_MAX_POLYS) {
    set_msg("tk_autotune: max_npoly out of range");
    return TK_ERR_INVALID_VALUE;
  }
  int rc = tk_init(device);
  if (rc) return rc;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  DeviceInfo* info;
  ensure_ready(device, &info);
  int16_t* buf = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&buf, max_npoly * 512u);
  if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, max_npoly * 512u);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double best_us[2][kBuckets];
  int best_v[2][kBuckets];
  const int top = size_bucket(max_npoly);
  for (int b = 0; b <= top && e == cudaSuccess; b++) {
    const size_t n = (size_t)1 << b;
    // enough launches per measurement for ~1 ms of work, at least 3
    int reps = (int)((size_t)(1u << 21) / n);
    reps = reps < 3 ? 3 : (reps > 200 ? 200 : reps);
    for (int dir = 0; dir < 2 && e == cudaSuccess; dir++) {
      best_us[dir][b] = 1e30;
      best_v[dir][b] = 0;
      for (int v = 0; v < tk::kNumMmaVariants && e == cudaSuccess; v++) {
        if (!tk::variant_valid(dir == 1, v)) continue;
        for (int w = 0; w < 2 && e == cudaSuccess; w++)
          e = tk::launch_mma(dir == 1, v, buf, buf, (long long)n, *info, st);
        if (e == cudaSuccess) e = cudaEventRecord(e0, st);
        for (int r = 0; r < reps && e == cudaSuccess; r++)
          e = tk::launch_mma(dir == 1, v, buf, buf, (long long)n, *info, st);
        if (e == cudaSuccess) e = cudaEventRecord(e1, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        const double us = 1e3 * ms / reps;
        if (e == cudaSuccess && us < best_us[dir][b]) {
          best_us[dir][b] = us;
          best_v[dir][b] = v;
        }
      }
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (buf) cudaFree(buf);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_err("tk_autotune", e);
    return TK_ERR_CUDA;
  }
  // Buckets above the tuned range inherit the largest tuned one.
  for (int dir = 0; dir < 2; dir++)
    for (int b = 0; b < kBuckets; b++) g_tuned[dir][b].store(best_v[dir][b <= top ? b : top]);
  if (cache_path) {
    FILE* f = fopen(cache_path, "w");
    if (f) {
      fprintf(f, "tk-autotune 1\n");
      for (int dir = 0; dir < 2; dir++)
        for (int b = 0; b <= top; b++)
          fprintf(f, "%d %d %d %.3f\n", dir, b, best_v[dir][b], best_us[dir][b]);
      fclose(f);
    }
  }
  return TK_SUCCESS;
}

int tk_autotune_reset(void) {
  for (auto& d : g_tuned)
    for (auto& b : d) b.store(-1);
  return TK_SUCCESS;
}

long long tk_get_table(int which, void* out, size_t bytes) {
  static tk::Matrices M;
  static tk::FwdFrags FF;
  static tk::InvFrags IF, IFR;
  static int32_t ZR[128];
  static uint8_t TC5[tk::kTc5TableBytes];
  static std::once_flag once;
  std::call_once(once, [] {
    tk::build_matrices(&M);
    tk::build_fwd_frags(M, &FF);
    tk::build_inv_frags(M, &IF);
    tk::build_pair_constants(ZR);
    tk::Matrices MR = M;
    tk::scale_inverse(&MR, 169);  // 2^-16 mod q
    tk::build_inv_frags(MR, &IFR);
    tk::build_tc5_tables(M, TC5);
  });
  const void* src;
  size_t size;
  switch (which) {
    case 0: src = M.m1; size = sizeof(M.m1); break;
    case 1: src = M.m2; size = sizeof(M.m2); break;
    case 2: src = M.ma; size = sizeof(M.ma); break;
    case 3: src = M.minv; size = sizeof(M.minv); break;
    case 4: src = &FF; size = sizeof(FF); break;
    case 5: src = &IF; size = sizeof(IF); break;
    case 6: src = ZR; size = sizeof(ZR); break;
    case 7: src = &IFR; size = sizeof(IFR); break;
    case 8: src = TC5; size = sizeof(TC5); break;
    default: return -TK_ERR_INVALID_VALUE;
  }
  if (out) memcpy(out, src, bytes < size ? bytes : size);
  return (long long)size;
}

}  // extern "C"
