/*
 * tk_ntt.h -- C ABI of the B200 batched ML-KEM NTT engine (libtk.so).
 *
 * Ring Z_3329[x]/(x^256+1), polynomials are int16_t[256], batches are npoly
 * contiguous polynomials (512 bytes each).  Conventions are those of the
 * pqcrystals reference that TensorKyber validates against:
 *
 *   forward  = ntt()    ntt_bench/ref/ntt.h:10-11, ntt_bench/ref/ntt.c:80-95
 *              standard-order input, bit-reversed output (128 degree-1
 *              residues mod X^2 - zeta as coefficient pairs), twiddles in
 *              Montgomery form so the output is in the normal domain.
 *   inverse  = invntt() ntt_bench/ref/ntt.h:13-14, ntt_bench/ref/ntt.c:106-126
 *              bit-reversed input, standard-order output, multiplied by the
 *              Montgomery factor 2^16 (invntt(ntt(x)) == 2^16 * x mod q).
 *
 * Every output coefficient is congruent mod q to the reference's output on the
 * same input.  The representatives are fixed and deterministic:
 *   forward output in [0, q), inverse output centred in [-(q-1)/2, (q-1)/2].
 * Both lie inside the bounds the reference's own outputs satisfy, so callers
 * that reduce afterwards (ML-KEM's poly_reduce) see identical residues.
 * Accepted inputs: any int16 (a superset of the inputs on which the
 * reference itself does not overflow int16: |x| <= 9471 for ntt(),
 * |x| <= 16383 for invntt()).
 *
 * Errors are returned as tk_status codes; no entry point exits or prints.
 * All entry points are thread-safe.  Device entry points are asynchronous on
 * the given stream (NULL = legacy default stream) and never allocate.
 */
#ifndef TK_NTT_H
#define TK_NTT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TK_ABI_VERSION 1

/* Same type as cudaStream_t; declared here so the header needs no CUDA headers. */
typedef struct CUstream_st *tk_stream_t;

typedef enum tk_status {
  TK_SUCCESS = 0,
  TK_ERR_INVALID_VALUE = 1,      /* NULL pointer, partially overlapping buffers, bad option */
  TK_ERR_MISALIGNED = 2,         /* polynomial buffer not 16-byte aligned */
  TK_ERR_TOO_LARGE = 3,          /* npoly above TK_MAX_POLYS */
  TK_ERR_NO_DEVICE = 4,          /* no CUDA device, or not an sm_100 (B200-class) GPU */
  TK_ERR_CUDA = 5,               /* a CUDA runtime call failed; tk_last_error() has the text */
  TK_ERR_NOT_DEVICE_MEMORY = 6,  /* device entry point given a pointer the GPU cannot address */
  TK_ERR_KERNEL_TIMEOUT = 7,     /* a kernel's bounded wait gave up (see tk_device_status) */
  TK_ERR_TIMEOUT = 8             /* a host-side wait reached its time limit */
} tk_status;

#define TK_MAX_POLYS ((size_t)1 << 32)

/* ---- device-memory batch transforms ------------------------------------
 * Replace the per-polynomial ntt()/invntt() (ntt_bench/ref/ntt.h:10-14) with
 * one call per batch, and the reference's in-place batch kernels
 * k_ntt_*(int16_t* d, int npoly) / k_invntt_*(int16_t* d, int npoly)
 * (ntt_bench/ntt_bench.cu:62, 98, 182, 231).  polys must be device (or
 * managed) memory, 16-byte aligned.  npoly == 0 is a successful no-op. */
int tk_ntt(int16_t *polys, size_t npoly, tk_stream_t stream);
int tk_invntt(int16_t *polys, size_t npoly, tk_stream_t stream);

/* Out-of-place forms: in and out are either identical or disjoint. */
int tk_ntt_oop(const int16_t *in, int16_t *out, size_t npoly, tk_stream_t stream);
int tk_invntt_oop(const int16_t *in, int16_t *out, size_t npoly, tk_stream_t stream);

/* ---- host-memory batch transforms (synchronous) -------------------------
 * Same contract as ntt()/invntt() applied to each polynomial of a host array
 * (ntt_bench/ref/ntt.h:10-14).  Copies in chunks through the current device
 * with copy/compute overlap; pinned host memory runs at full link speed. */
int tk_ntt_host(int16_t *polys, size_t npoly);
int tk_invntt_host(int16_t *polys, size_t npoly);

/* ---- small and packed forward inputs ---------------------------------------
 * Forward NTT of polynomials whose coefficients lie in [-128, 127] (ML-KEM
 * secrets and noise): stage 1 runs on one data byte per coefficient instead
 * of two (the reference's single-limb BASIC core,
 * ntt_bench/ntt_kernels.cuh:406-428).  in and out: device int16 rows, equal
 * (in place) or disjoint.  A coefficient outside the range sets
 * TK_FLAG_SMALL_RANGE (tk_device_status) and leaves that output unspecified.
 * Output as tk_ntt: NTT domain, [0, q). */
int tk_ntt_small(const int16_t *in, int16_t *out, size_t npoly, tk_stream_t stream);
/* Forward NTT of packed small polynomials (the reference's TC-PACK input,
 * ntt_bench/ntt_bench.cu:284-391): bits = 2 (64 bytes per polynomial,
 * coefficients in [-2, 1]) or 3 (128 bytes, [-4, 3]); coefficient i is the
 * two's-complement field at bit (i % (8/bits)) * bits of byte i / (8/bits).
 * packed: device memory, 16-byte aligned, not overlapping out. */
int tk_ntt_packed(const void *packed, int bits, int16_t *out, size_t npoly, tk_stream_t stream);
/* Host helper: packs npoly int16 polynomials into that format (packed must
 * hold npoly * 32 * bits bytes for bits = 2, npoly * 128 for bits = 3).
 * TK_ERR_INVALID_VALUE if a coefficient does not fit in `bits` bits. */
int tk_pack_small(const int16_t *polys, size_t npoly, int bits, void *packed);

/* ---- matrix-vector jobs (ML-KEM shape) ----------------------------------
 * For every job and i < k:
 *     out_i = invntt( sum_j basemul(A_ij, ntt(s_j)) ) + e_i       (mod q)
 * i.e. the composition of the reference's ntt (ntt_bench/ref/ntt.c:80-95),
 * basemul over the 128 coefficient pairs with +-zetas[64 + t/2]
 * (ntt_bench/ref/ntt.c:139-146) and invntt (ntt_bench/ref/ntt.c:106-126),
 * the product A^T r / A s of ML-KEM encryption and key generation.  The
 * reference repository has no polyvec wrapper; this call has no direct
 * counterpart there.  A is in the NTT domain; s, e any int16.  Output residues
 * are exact mod q; the representative is the centred inverse output plus e
 * (int16 wrap-around add, as the reference's polynomial add).
 * Jobs of one batch share k and are packed: job t uses A[t*k*k .. ),
 * s/e/out[t*k .. ).  Mixed ML-KEM-512/768/1024 work is one call with up to
 * three batches.  All buffers are device memory, 16-byte aligned; out may be
 * s itself but must not overlap A or e; e may be NULL.  Asynchronous on
 * stream; makes no allocation; capturable in a CUDA graph after tk_init. */
typedef struct tk_matvec_batch {
  int k;
  size_t njobs;
  const int16_t *A;
  const int16_t *s;
  const int16_t *e;
  int16_t *out;
} tk_matvec_batch;
int tk_matvec(const tk_matvec_batch *batches, int nbatches, tk_stream_t stream);
/* tk_matvec on HOST buffers, synchronous: copies A, s, e in (one copy when
 * they are contiguous, A then s then e), runs the same kernels, copies out
 * back (the plain per-request launch).  Uses a device
 * staging buffer per device that grows to the largest call (at most 8 GiB);
 * calls on one device are serialised.  out may alias s. */
int tk_matvec_host(const tk_matvec_batch *batches, int nbatches);
/* tk_matvec_host for callers that must not allocate (no counterpart in the
 * reference): services that reserve their device memory once at start-up and
 * may not grow it per request, and latency-bound paths that cannot take the
 * device-wide synchronisation of cudaFree or the cost of cudaMalloc and
 * stream creation.  Staging is a static device array of
 * TK_NOALLOC_SCRATCH_BYTES that comes with the library module (every GPU that
 * loads the library holds it until exit); a batch list needing more (A + s +
 * e + out bytes per batch, each rounded up to 256) returns TK_ERR_TOO_LARGE.
 * The work runs on `stream` and the call returns after synchronizing it; at
 * most 16 batches.  Per device, the first call looks up the array's address
 * (cudaGetSymbolAddress, with that device current): make it before any stream
 * capture.  The array keeps the last call's contents, which no call relies on;
 * calls on one device that overlap in time race on it. */
#define TK_NOALLOC_SCRATCH_BYTES (4 << 20)
int tk_matvec_host_noalloc(const tk_matvec_batch *batches, int nbatches, tk_stream_t stream);

/* ---- serving loop (continuous batching) ----------------------------------
 * A server runs matrix-vector jobs (tk_matvec semantics) from a device-
 * resident job ring through a persistent device loop.  tk_server_submit
 * queues a request of njobs jobs of one k whose buffers are HOST memory
 * (A: njobs*k*k, s/e/out: njobs*k polynomials; e may be NULL; A, s, e laid
 * out back to back travel in one copy; out may be s, must not overlap A or e).  Requests are admitted in arrival order as request slots (and, for staged requests, pool
 * memory) free up; their jobs run alongside jobs already on the GPU, and
 * results land in out before the ticket completes.
 *   - inputs: A, s, e are copied into the server's device pool of
 *     hbm_budget_bytes (admission waits for room), or, with zero_copy = 1
 *     and all three in page-locked host memory the device can address
 *     (cudaHostAlloc / cudaHostRegister), read in place over PCIe (uncached
 *     reads: slower than one bulk copy for all but tiny requests);
 *   - outputs: written in place when out is such memory (posted PCIe
 *     writes), else produced in the pool and copied back.
 * All host waits take a timeout; the device loop exits after
 * idle_exit_seconds without work and is relaunched on demand.  While it runs
 * it occupies every SM.  No reference counterpart (the reference times fixed
 * batches).  Buffers passed to submit must stay valid until the ticket
 * completes. */
typedef struct tk_server tk_server;
typedef struct tk_server_config {
  size_t hbm_budget_bytes;    /* device pool for staged requests (0: 1 GiB) */
  int max_inflight_requests;  /* request slots (0: 1024) */
  double idle_exit_seconds;   /* device loop idle limit (0: 0.02 s) */
  int zero_copy;              /* 1: read/write page-locked buffers in place */
} tk_server_config;
/* Cumulative counters; the *_ns sums split each completed request's latency
 * into queueing (submit -> admitted), device (admitted -> last job done) and
 * return (-> outputs in host memory) time. */
typedef struct tk_server_counters {
  unsigned long long requests_done, jobs_done, device_loop_launches;
  unsigned long long direct_requests, staged_requests;  /* inputs in place / staged */
  unsigned long long direct_outputs;                    /* outputs written in place */
  unsigned long long queue_ns, device_ns, return_ns;
  /* host-to-device copy operations issued for staged inputs: below
   * staged_requests when the inputs of requests admitted together lie back to
   * back in one page-locked allocation (they go in one copy) */
  unsigned long long input_copies;
} tk_server_counters;
int tk_server_create(int device, const tk_server_config *cfg, tk_server **out);
int tk_server_submit(tk_server *srv, int k, size_t njobs, const int16_t *A, const int16_t *s,
                     const int16_t *e, int16_t *out, uint64_t *ticket);
/* TK_SUCCESS once the request completed, TK_ERR_TIMEOUT if it has not. */
int tk_server_wait(tk_server *srv, uint64_t ticket, double timeout_s);
/* *done = 1 when complete; *latency_s = submit-to-completion time (or -1). */
int tk_server_query(tk_server *srv, uint64_t ticket, int *done, double *latency_s);
/* Forget a completed ticket. */
int tk_server_release(tk_server *srv, uint64_t ticket);
int tk_server_stats(tk_server *srv, tk_server_counters *out);
/* Waits (up to timeout_s) for outstanding requests, stops the loop, frees all. */
int tk_server_destroy(tk_server *srv, double timeout_s);

/* ---- process-wide options ---------------------------------------------------
 * TK_OPT_MATVEC_CHUNK_POLYS: vector polynomials per tk_matvec chunk (the
 * chunk's intermediates are meant to stay in L2); 0 restores the default.
 * TK_OPT_MATVEC_MODE: TK_MATVEC_PIPELINE (NTT, basemul-accumulate and iNTT+e
 * as three stream-ordered kernels per chunk), TK_MATVEC_FUSED (one kernel,
 * one warp per job: every intermediate stays in shared memory) or
 * TK_MATVEC_TILED (the default: one kernel for up to four batches, a CTA
 * carries a tile of 8 or 16 jobs through all three steps in shared memory).
 * TK_OPT_HOST_CHUNK_POLYS: largest number of polynomials per copy-in /
 * transform / copy-out chunk of tk_ntt_host / tk_invntt_host (1 .. 32768, the
 * default; smaller chunks are slower on a B200 host link: the path runs at the
 * link rate).  The first chunks of a call grow from 4096 polynomials to it and
 * the last ones shrink back, so the copies that cannot overlap stay short. */
#define TK_OPT_MATVEC_CHUNK_POLYS 1
#define TK_OPT_MATVEC_MODE 2
#define TK_OPT_HOST_CHUNK_POLYS 3
#define TK_MATVEC_PIPELINE 0
#define TK_MATVEC_FUSED 1
#define TK_MATVEC_TILED 2
int tk_set_option(int option, long long value);
long long tk_get_option(int option);

/* ---- runtime --------------------------------------------------------------
 * tk_init: per-device set-up (constant tables, occupancy).  Every entry point
 * runs it on first use of a device; call it explicitly before capturing a
 * CUDA graph, because the set-up makes synchronous copies.  Corresponds to
 * the reference's cudaMemcpyToSymbol(d_zetas) + setup_tc_matrices()
 * (ntt_bench/ntt_bench.cu:932-933, ntt_bench/ntt_kernels.cuh:842-925). */
int tk_init(int device);

/* Reads and clears the kernel-side error flags of a device (bit 0: forward,
 * bit 1: inverse kernel gave up on a bounded wait; bit 2: tk_ntt_small saw a
 * coefficient outside [-128, 127]; bit 3: tk_selftest_bounded_wait; bit 4:
 * the TK_MATVEC_TILED kernel gave up on a bounded wait).
 * Synchronous. */
#define TK_FLAG_FORWARD_TIMEOUT 1u
#define TK_FLAG_INVERSE_TIMEOUT 2u
#define TK_FLAG_SMALL_RANGE 4u
#define TK_FLAG_SELFTEST_TIMEOUT 8u
#define TK_FLAG_MATVEC_TIMEOUT 16u
int tk_device_status(int device, unsigned *flags);
/* Exercises the kernels' give-up path: one CTA waits on an mbarrier that
 * nothing completes, through the same bounded wait as the batch kernels, and
 * after `seconds` (0 < seconds <= 10) sets TK_FLAG_SELFTEST_TIMEOUT and
 * returns; the context stays usable.  Synchronous.  No reference counterpart. */
int tk_selftest_bounded_wait(int device, double seconds);

/* ---- kernel variants ------------------------------------------------------
 * The engine ships several kernel variants (CTA shape, pipeline depth) and
 * picks one per direction and batch size.  tk_set_variant forces one for all
 * later calls in the process (-1 restores automatic choice); tk_get_variant
 * reports the choice for a batch size.  No reference counterpart: the
 * reference binary times each of its variants from main()
 * (ntt_bench/ntt_bench.cu:967-974). */
#define TK_FORWARD 0
#define TK_INVERSE 1
int tk_variant_count(void);
const char *tk_variant_name(int variant);
int tk_set_variant(int direction, int variant);
int tk_get_variant(int direction, size_t npoly);

/* Autotuner.  Times every variant in both directions at each power-of-two
 * batch size 1 .. max_npoly on `device` (one scratch buffer of max_npoly
 * polynomials is allocated and freed) and keeps the fastest per direction and
 * size bucket floor(log2(npoly)) for all later calls; larger sizes use the
 * largest tuned bucket.  With cache_path, a valid cache file is loaded instead
 * of tuning, and a fresh tuning is written to it.  Synchronous.
 * tk_autotune_reset() returns to the built-in choice. */
int tk_autotune(int device, size_t max_npoly, const char *cache_path);
int tk_autotune_reset(void);

const char *tk_status_string(int status);
/* Detail of the last failure on the calling thread ("" if none). */
const char *tk_last_error(void);
int tk_abi_version(void);

/* ---- constant tables (no GPU needed) -------------------------------------
 * The host matrix builder's output, for inspection and tests.  which:
 *   0: M1[16][16]   1: M2[16][16][16]   2: MA[16][16][16]   3: Minv[16][16]
 *      (int16 residues in [0, q), see tensorkyber_b200/csrc/tk_tables.h)
 *   4: forward fragment tables   5: inverse fragment tables
 *   6: basemul pair constants int32[128], z_t * 2^-16 mod q with
 *      z_t = +-17^brv7(64 + t/2) (+ for even t), as the matrix-vector
 *      kernels upload them
 *   7: the tiled matrix-vector kernel's inverse fragment tables (layout of
 *      5), computing 2^-16 * invntt
 *   8: the tcgen05 kernels' 68 int8 B-operand tiles of 1 KiB (tcgen05 K-major
 *      layout; see tensorkyber_b200/csrc/tk_tables.h)
 * Copies min(bytes, size) bytes to out and returns the table size in bytes,
 * or -TK_ERR_INVALID_VALUE.  Counterpart of setup_tc_matrices
 * (ntt_bench/ntt_kernels.cuh:842-925), which builds the same maps. */
long long tk_get_table(int which, void *out, size_t bytes);

#ifdef __cplusplus
}
#endif
#endif /* TK_NTT_H */
