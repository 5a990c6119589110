// tk_internal.h -- declarations shared between the kernel translation units and
// the C ABI layer (tk_api.cu).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tk {

// Kernel variants.  mma.sync (CTA shape / pipeline depth):
//   0: 4 warps, 32-polynomial tiles, 3 slots   (4 CTAs/SM)
//   1: 8 warps, 64-polynomial tiles, 3 slots   (2 CTAs/SM)
//   2: 4 warps, 32-polynomial tiles, 2 slots   (6 CTAs/SM)
//   3: 4 warps, 32-polynomial tiles, 2 slots, forward stage 1 kept as int32
//      sums in a shared-memory tile (3 CTAs/SM)
// tcgen05:
//   4: 128-polynomial tiles, tcgen05.mma kind::i8 with tensor-memory
//      accumulators, the second stage's operand in tensor memory (tk_tc5.cu;
//      1 CTA/SM)
constexpr int kNumMmaSyncVariants = 4;
constexpr int kTc5Variant = 4;
constexpr int kNumMmaVariants = 5;
inline bool variant_valid(bool /*inverse*/, int v) { return v >= 0 && v < kNumMmaVariants; }
// Largest batch one kernel launch covers (TMA coordinates are signed 32-bit).
constexpr long long kMaxLaunchPolys = 1ll << 30;

// Forward input forms besides int16: 1 = int16 with coefficients in
// [-128, 127], 2 / 3 = packed 2- / 3-bit fields (single-limb stage 1).
constexpr int kNumInputForms = 3;

struct DeviceInfo {
  int device = -1;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  int mma_ctas_per_sm[2][kNumMmaSyncVariants] = {{1, 1, 1, 1}, {1, 1, 1, 1}};  // [inverse][variant]
  int form_ctas_per_sm[kNumInputForms] = {1, 1, 1};  // forward input forms 1..3
  int add_ctas_per_sm[kNumMmaSyncVariants] = {1, 1, 1, 1};  // inverse with addend
  int multi_ctas_per_sm[3] = {1, 1, 1};  // multi-segment forward / inverse / inverse+addend
  int tile_ctas_per_sm = 1;              // k_matvec_tiles
  size_t total_mem = 0;
  unsigned* status = nullptr;            // the device's kernel status flags (device address)
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

// One batch of a multi-batch launch: npoly polynomials src -> dst (src == dst
// for in place); inverse only: an optional addend.
struct Seg {
  const int16_t* src;
  int16_t* dst;
  long long npoly;
  const int16_t* addend;
};
constexpr int kMaxSegs = 4;  // batches per kernel launch
// Transforms every segment, packing up to kMaxSegs of them (pieces of at
// most kMaxLaunchPolys) into each kernel launch, so several small batches
// fill the GPU like one large one.  A launch of one piece uses the given
// variant's single-batch kernel; a launch of several uses the default
// variants' shapes (forward 3, inverse 0).  A segment with an addend selects
// the inverse-with-addend kernel for its launch (segments without one add
// nothing).
cudaError_t launch_mma_segs(bool inverse, int variant, const Seg* segs, int nseg,
                            const DeviceInfo& info, cudaStream_t stream);

// CUresult of the calling thread's last tensor-map encode (launch_mma reports
// cudaErrorInvalidResourceHandle when an encode failed); note_encode_result
// records one from another unit.
int last_encode_result();
void note_encode_result(int r);

// The tcgen05 kernels (tk_tc5.cu): per-device set-up (constant tiles, shared
// memory limits) and the batched transform src -> dst (src == dst in place).
bool tc5_init_device(DeviceInfo* info);
cudaError_t launch_tc5(bool inverse, const int16_t* src, int16_t* dst, long long npoly,
                       const DeviceInfo& info, cudaStream_t stream);

// Matrix-vector jobs (tk_matvec.cu).  Chunks hold at most this many vector
// polynomials, so that intermediates stay in the 126 MB L2.
constexpr long long kMatvecChunkVecPolys = 131072;  // default (64 MiB); tk_set_option may change it
bool matvec_init_device();
// Up to three uniform-k batches for the single-launch fused kernel: global job
// g belongs to batch b when first[b] <= g < first[b+1]; gfirst is the same
// prefix over work items of floor(8 / k) jobs (filled by launch_matvec_fused).
struct FusedBatches {
  int nb;
  int k[3];
  int first[4];
  int gfirst[4];
  const int16_t* A[3];
  const int16_t* s[3];
  const int16_t* e[3];
  int16_t* out[3];
};
cudaError_t launch_matvec_fused(const FusedBatches& args, const DeviceInfo& info,
                                cudaStream_t stream);
// One uniform-k batch of device buffers for the three-kernel pipeline.
struct MatvecPart {
  int k;
  size_t njobs;
  const int16_t* A;
  const int16_t* s;
  const int16_t* e;
  int16_t* out;
};
// The pipeline over up to kMaxSegs batches (forward NTT, basemul-accumulate,
// inverse NTT + e per chunk of at most chunk_vec_polys vector polynomials).
cudaError_t launch_matvec(const MatvecPart* batches, int nb, const DeviceInfo& info,
                          cudaStream_t stream, int fwd_variant, int inv_variant,
                          long long chunk_vec_polys);
// The tiled single-kernel form: one k_matvec_tiles launch for up to kMaxSegs
// batches (forward NTT, basemul-accumulate and inverse NTT + e of a tile of
// jobs in one CTA's shared memory).
cudaError_t launch_matvec_tile(const MatvecPart* batches, int nb, const DeviceInfo& info,
                               cudaStream_t stream);

// ---- serving loop (device side in tk_matvec.cu, host side in tk_serve.cpp) ----
// One job descriptor of the job ring (64 bytes; the ring lives in mapped
// page-locked host memory).
struct alignas(64) ServeJob {
  const int16_t* A;
  const int16_t* s;
  const int16_t* e;
  int16_t* out;
  uint32_t k;
  uint32_t req;    // request slot
  uint32_t njobs;  // jobs of the request
  uint32_t gen;    // request generation written to the completion flag
  uint64_t pad[2];
};
// Device-memory control block, one 128-byte line per writer: head (claimed
// jobs, device compare-and-swap), then the host-written words (tail =
// published jobs, stream-written; stop) with the device's closing flag, then
// the time of the latest claim.  head and tail count modulo 2^32 and are
// compared as (int)(tail - head).
struct alignas(128) ServeCtl {
  unsigned int head;  // next job to claim (device compare-and-swap)
  unsigned int pad0[31];
  unsigned int tail;     // jobs published (host)
  unsigned int stop;     // host: end the loop now
  unsigned int closing;  // device: the loop is leaving (host clears)
  unsigned int pad1[29];
  unsigned long long last_claim_ns;  // globaltimer of the latest claim
  unsigned long long pad2[15];
};
// Launches the persistent serving kernel.  ring: the job ring (mapped host
// memory); req_ctr: per-slot done counters (device memory); req_flag: per-slot
// completion flags in mapped pinned host memory; idle_ns: the loop exits after
// this long without a claim anywhere.
cudaError_t launch_serve(const ServeJob* ring, uint32_t ring_mask, ServeCtl* ctl,
                         unsigned int* req_ctr, unsigned int* req_flag, unsigned long long idle_ns,
                         const DeviceInfo& info, cudaStream_t stream);

// Per-device state of the API layer (set-up on first use), for other units.
int api_device_info(int device, DeviceInfo** info);

// True when one host<->device copy may cover host bytes [p, p + bytes): the
// range starts in pageable memory, or lies inside one page-locked
// allocation (a copy that runs from one page-locked allocation into the next
// is not valid).  Needs the device's context current on the calling thread.
bool host_span_one_copy(const void* p, size_t bytes);

// Forward transform of npoly polynomials given in input form `form` (1..3):
// src holds int16 rows (form 1; src == dst for in place) or packed rows of
// 64 / 128 bytes (forms 2 / 3); dst gets int16 NTT-domain rows in [0, q).
// Form 1 sets status bit 2 when an input lies outside [-128, 127].
cudaError_t launch_fwd_form(int form, const void* src, int16_t* dst, long long npoly,
                            const DeviceInfo& info, cudaStream_t stream);

// One CTA that lets a bounded mbarrier wait run out (status bit 3).
cudaError_t launch_selftest_wait(unsigned long long limit_ns, cudaStream_t stream);

// Kernel-side error flags (bounded waits that gave up), read and reset.
cudaError_t read_and_clear_status(unsigned* flags);

}  // namespace tk
