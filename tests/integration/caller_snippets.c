/* The C calls a reference-side caller makes into libtk.so, as functions over
 * the variables such a caller holds.  Compiled against include/ with warnings
 * as errors and linked against libtk.so by tests/test_integration_snippets.py
 * (nothing is executed).  Reference call sites they replace:
 *   batch kernels  k_ntt_* / k_invntt_*(d_buf, npoly)  ntt_bench/ntt_bench.cu:616, 620
 *   TC-PACK input                                       ntt_bench/ntt_bench.cu:284-391 */
#include <stdint.h>
#include <stdio.h>

#include "tk_ntt.h"

/* Batched calls from the reference's CUDA harness, in place on a device buffer. */
int batched_in_place(int16_t *d_buf, int npoly, tk_stream_t stream) {
  int rc = tk_ntt(d_buf, (size_t)npoly, (tk_stream_t)stream); /* was k_ntt_*<<<>>>   */
  if (rc != TK_SUCCESS) fprintf(stderr, "%s: %s\n", tk_status_string(rc), tk_last_error());
  rc = tk_invntt(d_buf, (size_t)npoly, (tk_stream_t)stream); /* was k_invntt_*<<<>>> */
  return rc;
}

/* Small, packed and matrix-vector inputs. */
int small_packed_matvec(int16_t *d_s, int npoly, tk_stream_t stream, const int16_t *h_polys,
                        void *h_packed, const void *d_packed, int16_t *d_out, size_t n2,
                        size_t n3, size_t n4, const int16_t *A2, const int16_t *A3,
                        const int16_t *A4, const int16_t *s2, const int16_t *s3,
                        const int16_t *s4, const int16_t *e2, const int16_t *e3,
                        const int16_t *e4, int16_t *out2, int16_t *out3, int16_t *out4) {
  /* ML-KEM secrets / noise (coefficients in [-128, 127]): single-limb stage 1 */
  tk_ntt_small(d_s, d_s, (size_t)npoly, stream); /* in place */
  /* TC-PACK input: 64 B (2-bit) per polynomial */
  tk_pack_small(h_polys, (size_t)npoly, 2, h_packed); /* host packing helper */
  tk_ntt_packed(d_packed, 2, d_out, (size_t)npoly, stream);
  /* out_i = invntt(sum_j A_ij o ntt(s_j)) + e_i, mixed k in one call */
  tk_matvec_batch b[3] = {{2, n2, A2, s2, e2, out2}, {3, n3, A3, s3, e3, out3},
                          {4, n4, A4, s4, e4, out4}};
  return tk_matvec(b, 3, stream);
}

/* Callers that may not allocate: staging in the library's static scratch. */
int no_alloc_matvec(const tk_matvec_batch *batches, int nbatches, tk_stream_t stream) {
  return tk_matvec_host_noalloc(batches, nbatches, stream);
}

/* Serving (continuous batching) on host buffers. */
int serving(int k, size_t njobs, const int16_t *h_A, const int16_t *h_s, const int16_t *h_e,
            int16_t *h_out) {
  tk_server *srv;
  tk_server_config cfg = {0}; /* 1 GiB pool, 1024 slots, 20 ms idle exit */
  int rc = tk_server_create(0, &cfg, &srv);
  if (rc != TK_SUCCESS) return rc;
  uint64_t t;
  tk_server_submit(srv, k, njobs, h_A, h_s, h_e, h_out, &t); /* host buffers */
  tk_server_wait(srv, t, 1.0); /* TK_ERR_TIMEOUT if not done in 1 s */
  tk_server_release(srv, t);
  return tk_server_destroy(srv, 10.0);
}
