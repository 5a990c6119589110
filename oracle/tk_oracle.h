/*
 * tk_oracle.h -- CPU restatement of the reference NTT path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity checker for the GPU engine: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may
 * load it.  The shipped library (tensorkyber_b200/) never links or calls it.
 *
 * Every function restates the pqcrystals reference code that TensorKyber
 * validates against (file:line below are paths inside the TensorKyber repo):
 *
 *   tko_montgomery_reduce   ntt_bench/ref/reduce.c:16-23  (QINV = -3327, reduce.h:8)
 *   tko_barrett_reduce      ntt_bench/ref/reduce.c:35-42
 *   tko_fqmul               ntt_bench/ref/ntt.c:68-70
 *   tko_zetas               ntt_bench/ref/ntt.c:39-56 (generated here from the
 *                           definition in the comment at ntt.c:5-37, not copied)
 *   tko_ntt                 ntt_bench/ref/ntt.c:80-95
 *   tko_invntt              ntt_bench/ref/ntt.c:106-126
 *   tko_basemul             ntt_bench/ref/ntt.c:139-146
 *
 * Parity is pinned by tests/test_oracle.py against the reference's own C
 * sources compiled unmodified into oracle/_ref/ (see oracle/Makefile) and
 * against the committed fixtures in tests/golden/.
 */
#ifndef TK_ORACLE_H
#define TK_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TKO_N 256
#define TKO_Q 3329

/* twiddles: zetas[i] = centre(2^16 * 17^brv7(i) mod q) */
extern int16_t tko_zetas[128];
void tko_init(void); /* fills tko_zetas; idempotent, called by every entry */

int16_t tko_montgomery_reduce(int32_t a);
int16_t tko_barrett_reduce(int16_t a);
int16_t tko_fqmul(int16_t a, int16_t b);

void tko_ntt(int16_t r[256]);
void tko_invntt(int16_t r[256]);
void tko_basemul(int16_t r[2], const int16_t a[2], const int16_t b[2], int16_t zeta);

/* Batched forms: polys is npoly contiguous int16[256]. */
void tko_ntt_batch(int16_t *polys, size_t npoly);
void tko_invntt_batch(int16_t *polys, size_t npoly);

/* Pointwise product of two NTT-domain polys, the standard ML-KEM composition of
 * basemul over the 128 degree-1 residues: pair i uses +zetas[64+i/2] for even i
 * and -zetas[64+i/2] for odd i. */
void tko_poly_basemul(int16_t r[256], const int16_t a[256], const int16_t b[256]);

/* One fused matrix-vector job of the ML-KEM encryption shape:
 *   s_hat[j] = ntt(s[j]);  acc[i] = barrett(sum_j poly_basemul(A[i][j], s_hat[j]));
 *   out[i]   = invntt(acc[i]) + e[i]
 * A is k*k polys (row-major, already in the NTT domain), s, e and out are k polys. */
void tko_matvec_job(int k, const int16_t *A, const int16_t *s, const int16_t *e,
                    int16_t *out);

/* Canonical residue in [0, q). */
static inline int16_t tko_canon(int32_t v)
{
  int32_t t = v % TKO_Q;
  return (int16_t)(t < 0 ? t + TKO_Q : t);
}

/* CPU throughput harness.  Runs fwd() then inv() on every poly of a private
 * copy of `src` (npoly polys) per thread, repeating until at least min_seconds
 * of wall time has passed.  Function pointers let the same harness time the
 * reference's own symbols (oracle/_ref) or this restatement.  Returns polys/s
 * of complete NTT+iNTT round trips summed over all threads; *polys_done gets
 * the number of round trips executed. */
typedef void (*tko_poly_fn)(int16_t *);
double tko_time_roundtrip(tko_poly_fn fwd, tko_poly_fn inv, const int16_t *src,
                          size_t npoly, int threads, double min_seconds,
                          uint64_t *polys_done);

/* Packed small-coefficient polynomials (the TC-PACK input format): `bits`-bit
 * two's-complement fields, 8/bits coefficients per byte, coefficient i in
 * byte i/(8/bits) at bit (i % (8/bits))*bits.  tko_pack_small restates the
 * reference harness's pack_small (ntt_bench/ntt_bench.cu:744-752) and returns
 * the bytes per polynomial; tko_unpack_small restates the kernel's unpacking
 * with sign extension (ntt_bench/ntt_bench.cu:317-340).  bits is 2 or 3. */
size_t tko_pack_small(int bits, const int16_t poly[256], uint8_t *packed);
void tko_unpack_small(int bits, const uint8_t *packed, int16_t poly[256]);

/* One pass: polys (npoly, in place) is split into `threads` contiguous
 * chunks and each thread applies fwd() then inv() to every poly of its chunk.
 * Returns the wall time in seconds (negative on failure). */
double tko_split_roundtrip(tko_poly_fn fwd, tko_poly_fn inv, int16_t *polys, size_t npoly,
                           int threads);

#ifdef __cplusplus
}
#endif
#endif
