/*
 * tk_pqcrystals.h -- link-compatible replacements for the reference's
 * per-polynomial transforms (libtk_pqcrystals.so).
 *
 * The reference declares void ntt(int16_t poly[256]) and
 * void invntt(int16_t poly[256]) (ntt_bench/ref/ntt.h:10-14), renamed by
 * KYBER_NAMESPACE to pqcrystals_kyber{512,768,1024}_ref_{ntt,invntt}
 * (ntt_bench/ref/params.h:10-18).  These exports carry exactly those names, so
 * a program linked against ref/ntt.o can link against this library instead.
 * Each call transforms one host polynomial through tk_ntt_host/tk_invntt_host
 * (a device round trip per call: for throughput, call the batched tk_* entry
 * points of tk_ntt.h instead).  Output residues equal the reference's mod q;
 * representatives are tk_ntt.h's ([0, q) forward, centred inverse).  The
 * reference functions return void, so a failure cannot be reported through
 * them: on error the polynomial is left unchanged and the status is kept
 * for tk_pqcrystals_last_status().
 */
#ifndef TK_PQCRYSTALS_H
#define TK_PQCRYSTALS_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

void pqcrystals_kyber512_ref_ntt(int16_t poly[256]);
void pqcrystals_kyber512_ref_invntt(int16_t poly[256]);
void pqcrystals_kyber768_ref_ntt(int16_t poly[256]);
void pqcrystals_kyber768_ref_invntt(int16_t poly[256]);
void pqcrystals_kyber1024_ref_ntt(int16_t poly[256]);
void pqcrystals_kyber1024_ref_invntt(int16_t poly[256]);

/* tk_status of the calling thread's last shim call (0 = success). */
int tk_pqcrystals_last_status(void);

#ifdef __cplusplus
}
#endif
#endif
