/* tk_pqcrystals_shim.c -- the reference's per-polynomial symbol names
 * (ntt_bench/ref/ntt.h:10-14 under the KYBER_NAMESPACE renaming of
 * ntt_bench/ref/params.h:10-18) forwarded to the batched GPU engine. */
#include <string.h>

#include "../../include/tk_ntt.h"
#include "../../include/tk_pqcrystals.h"

static _Thread_local int last_status = 0;

static void run(int16_t poly[256], int inverse)
{
  int16_t tmp[256];
  memcpy(tmp, poly, sizeof(tmp));
  last_status = inverse ? tk_invntt_host(tmp, 1) : tk_ntt_host(tmp, 1);
  if (last_status == TK_SUCCESS) memcpy(poly, tmp, sizeof(tmp));
}

void pqcrystals_kyber512_ref_ntt(int16_t poly[256]) { run(poly, 0); }
void pqcrystals_kyber512_ref_invntt(int16_t poly[256]) { run(poly, 1); }
void pqcrystals_kyber768_ref_ntt(int16_t poly[256]) { run(poly, 0); }
void pqcrystals_kyber768_ref_invntt(int16_t poly[256]) { run(poly, 1); }
void pqcrystals_kyber1024_ref_ntt(int16_t poly[256]) { run(poly, 0); }
void pqcrystals_kyber1024_ref_invntt(int16_t poly[256]) { run(poly, 1); }

int tk_pqcrystals_last_status(void) { return last_status; }
