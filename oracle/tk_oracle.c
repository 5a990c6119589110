/*
 * tk_oracle.c -- CPU restatement of the pqcrystals reference NTT used by
 * TensorKyber as its ground truth.  TEST INFRASTRUCTURE ONLY (see tk_oracle.h):
 * the GPU library never links this file.
 *
 * Integer semantics follow the reference exactly, including the int16
 * truncations that C performs on assignment; casts are spelled out so the
 * wrap-around is explicit rather than implementation-defined.
 */
#include "tk_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define TKO_QINV (-3327)                 /* q^-1 mod 2^16, ref/reduce.h:8      */
#define TKO_MONT (-1044)                 /* 2^16 mod q (centred), ref/reduce.h:7 */
#define TKO_INV_F 1441                   /* mont^2/128, ref/ntt.c:109           */

int16_t tko_zetas[128];
static int tko_ready = 0;

static inline int16_t wrap16(int32_t v) { return (int16_t)(uint16_t)(uint32_t)v; }

/* ref/reduce.c:16-23: t = (int16)a * QINV; return (a - t*q) >> 16 */
int16_t tko_montgomery_reduce(int32_t a)
{
  int16_t t = wrap16((int32_t)wrap16(a) * TKO_QINV);
  return wrap16((a - (int32_t)t * TKO_Q) >> 16);
}

/* ref/reduce.c:35-42: centred Barrett, v = round(2^26/q) = 20159 */
int16_t tko_barrett_reduce(int16_t a)
{
  const int32_t v = ((1 << 26) + TKO_Q / 2) / TKO_Q;
  int16_t t = wrap16(((int32_t)v * a + (1 << 25)) >> 26);
  t = wrap16((int32_t)t * TKO_Q);
  return wrap16((int32_t)a - t);
}

/* ref/ntt.c:68-70 */
int16_t tko_fqmul(int16_t a, int16_t b) { return tko_montgomery_reduce((int32_t)a * b); }

static unsigned brv7(unsigned x)
{
  unsigned r = 0;
  for (int b = 0; b < 7; b++) r |= ((x >> b) & 1u) << (6 - b);
  return r;
}

/* The table at ref/ntt.c:39-56 is defined (ntt.c:5-37) as
 * zetas[i] = 2^16 * 17^brv7(i) mod q, brought into [-(q-1)/2, (q-1)/2].
 * It is recomputed here from that definition with plain modular powers. */
void tko_init(void)
{
  if (tko_ready) return;
  for (unsigned i = 0; i < 128; i++) {
    uint32_t e = brv7(i), acc = 1, base = 17;
    while (e) {
      if (e & 1u) acc = (acc * base) % TKO_Q;
      base = (base * base) % TKO_Q;
      e >>= 1;
    }
    int32_t z = (int32_t)((acc * 65536u) % TKO_Q);
    if (z > TKO_Q / 2) z -= TKO_Q;
    tko_zetas[i] = (int16_t)z;
  }
  tko_ready = 1;
}

/* ref/ntt.c:80-95: Cooley-Tukey, len 128 -> 2, zetas[1..127] in order. */
void tko_ntt(int16_t r[256])
{
  tko_init();
  unsigned k = 1;
  for (unsigned len = 128; len >= 2; len >>= 1) {
    for (unsigned start = 0; start < 256; start += 2 * len) {
      const int16_t zeta = tko_zetas[k++];
      for (unsigned j = start; j < start + len; j++) {
        const int16_t t = tko_fqmul(zeta, r[j + len]);
        r[j + len] = wrap16((int32_t)r[j] - t);
        r[j] = wrap16((int32_t)r[j] + t);
      }
    }
  }
}

/* ref/ntt.c:106-126: Gentleman-Sande, len 2 -> 128, zetas[127..1], Barrett on
 * the sums, then multiply every coefficient by 1441 (Montgomery). */
void tko_invntt(int16_t r[256])
{
  tko_init();
  unsigned k = 127;
  for (unsigned len = 2; len <= 128; len <<= 1) {
    for (unsigned start = 0; start < 256; start += 2 * len) {
      const int16_t zeta = tko_zetas[k--];
      for (unsigned j = start; j < start + len; j++) {
        const int16_t t = r[j];
        r[j] = tko_barrett_reduce(wrap16((int32_t)t + r[j + len]));
        r[j + len] = wrap16((int32_t)r[j + len] - t);
        r[j + len] = tko_fqmul(zeta, r[j + len]);
      }
    }
  }
  for (unsigned j = 0; j < 256; j++) r[j] = tko_fqmul(r[j], TKO_INV_F);
}

/* ref/ntt.c:139-146 */
void tko_basemul(int16_t r[2], const int16_t a[2], const int16_t b[2], int16_t zeta)
{
  int16_t r0 = tko_fqmul(a[1], b[1]);
  r0 = tko_fqmul(r0, zeta);
  r0 = wrap16((int32_t)r0 + tko_fqmul(a[0], b[0]));
  int16_t r1 = tko_fqmul(a[0], b[1]);
  r1 = wrap16((int32_t)r1 + tko_fqmul(a[1], b[0]));
  r[0] = r0;
  r[1] = r1;
}

void tko_ntt_batch(int16_t *polys, size_t npoly)
{
  for (size_t i = 0; i < npoly; i++) tko_ntt(polys + i * TKO_N);
}

void tko_invntt_batch(int16_t *polys, size_t npoly)
{
  for (size_t i = 0; i < npoly; i++) tko_invntt(polys + i * TKO_N);
}

void tko_poly_basemul(int16_t r[256], const int16_t a[256], const int16_t b[256])
{
  tko_init();
  for (unsigned i = 0; i < 64; i++) {
    tko_basemul(r + 4 * i, a + 4 * i, b + 4 * i, tko_zetas[64 + i]);
    tko_basemul(r + 4 * i + 2, a + 4 * i + 2, b + 4 * i + 2, (int16_t)-tko_zetas[64 + i]);
  }
}

void tko_matvec_job(int k, const int16_t *A, const int16_t *s, const int16_t *e,
                    int16_t *out)
{
  int16_t shat[4][TKO_N], acc[TKO_N], t[TKO_N];
  for (int j = 0; j < k; j++) {
    memcpy(shat[j], s + (size_t)j * TKO_N, sizeof(shat[j]));
    tko_ntt(shat[j]);
  }
  for (int i = 0; i < k; i++) {
    tko_poly_basemul(acc, A + ((size_t)i * k) * TKO_N, shat[0]);
    for (int j = 1; j < k; j++) {
      tko_poly_basemul(t, A + ((size_t)i * k + j) * TKO_N, shat[j]);
      for (int c = 0; c < TKO_N; c++) acc[c] = wrap16((int32_t)acc[c] + t[c]);
    }
    for (int c = 0; c < TKO_N; c++) acc[c] = tko_barrett_reduce(acc[c]);
    tko_invntt(acc);
    for (int c = 0; c < TKO_N; c++)
      out[(size_t)i * TKO_N + c] = wrap16((int32_t)acc[c] + e[(size_t)i * TKO_N + c]);
  }
}

/* ---------------------------------------------------------------- timing -- */

typedef struct {
  tko_poly_fn fwd, inv;
  const int16_t *src;
  size_t npoly;
  double min_seconds;
  uint64_t done;
  int err;
} tko_job;

static double now_s(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void *tko_worker(void *arg)
{
  tko_job *j = (tko_job *)arg;
  int16_t *buf = (int16_t *)malloc(j->npoly * TKO_N * sizeof(int16_t));
  if (!buf) {
    j->err = 1;
    return NULL;
  }
  memcpy(buf, j->src, j->npoly * TKO_N * sizeof(int16_t));
  const double t0 = now_s();
  uint64_t done = 0;
  do {
    /* ntt output is un-reduced but |v| < 8q; invntt output is in (-q, q), so
     * repeating the round trip in place stays inside the reference's domain */
    for (size_t i = 0; i < j->npoly; i++) {
      j->fwd(buf + i * TKO_N);
      j->inv(buf + i * TKO_N);
    }
    done += j->npoly;
  } while (now_s() - t0 < j->min_seconds);
  j->done = done;
  free(buf);
  return NULL;
}

double tko_time_roundtrip(tko_poly_fn fwd, tko_poly_fn inv, const int16_t *src,
                          size_t npoly, int threads, double min_seconds,
                          uint64_t *polys_done)
{
  if (threads < 1) threads = 1;
  if (threads > 1024) threads = 1024;
  tko_job *jobs = (tko_job *)calloc((size_t)threads, sizeof(tko_job));
  pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
  if (!jobs || !tid) {
    free(jobs);
    free(tid);
    return -1.0;
  }
  const double t0 = now_s();
  for (int i = 0; i < threads; i++) {
    jobs[i] = (tko_job){fwd, inv, src, npoly, min_seconds, 0, 0};
    pthread_create(&tid[i], NULL, tko_worker, &jobs[i]);
  }
  uint64_t total = 0;
  int err = 0;
  for (int i = 0; i < threads; i++) {
    pthread_join(tid[i], NULL);
    total += jobs[i].done;
    err |= jobs[i].err;
  }
  const double dt = now_s() - t0;
  free(jobs);
  free(tid);
  if (polys_done) *polys_done = total;
  if (err || dt <= 0) return -1.0;
  return (double)total / dt;
}

typedef struct {
  tko_poly_fn fwd, inv;
  int16_t *polys;
  size_t n;
} tko_chunk;

static void *tko_chunk_worker(void *arg)
{
  tko_chunk *c = (tko_chunk *)arg;
  for (size_t i = 0; i < c->n; i++) {
    c->fwd(c->polys + i * TKO_N);
    c->inv(c->polys + i * TKO_N);
  }
  return NULL;
}

double tko_split_roundtrip(tko_poly_fn fwd, tko_poly_fn inv, int16_t *polys, size_t npoly,
                           int threads)
{
  if (threads < 1) threads = 1;
  if ((size_t)threads > npoly) threads = (int)(npoly ? npoly : 1);
  tko_chunk *cs = (tko_chunk *)calloc((size_t)threads, sizeof(tko_chunk));
  pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
  if (!cs || !tid) {
    free(cs);
    free(tid);
    return -1.0;
  }
  const double t0 = now_s();
  size_t start = 0;
  for (int i = 0; i < threads; i++) {
    const size_t n = npoly / (size_t)threads + ((size_t)i < npoly % (size_t)threads ? 1 : 0);
    cs[i] = (tko_chunk){fwd, inv, polys + start * TKO_N, n};
    start += n;
    pthread_create(&tid[i], NULL, tko_chunk_worker, &cs[i]);
  }
  for (int i = 0; i < threads; i++) pthread_join(tid[i], NULL);
  const double dt = now_s() - t0;
  free(cs);
  free(tid);
  return dt;
}

/* ntt_bench/ntt_bench.cu:744-752: per = 8/bits fields per byte, low bits first. */
size_t tko_pack_small(int bits, const int16_t poly[256], uint8_t *packed) {
  const int per = 8 / bits;
  const size_t nbytes = (256 + per - 1) / per;
  memset(packed, 0, nbytes);
  for (int i = 0; i < 256; i++)
    packed[i / per] |= (uint8_t)((poly[i] & ((1 << bits) - 1)) << ((i % per) * bits));
  return nbytes;
}

/* ntt_bench/ntt_bench.cu:317-340: the field, sign-extended from `bits` bits. */
void tko_unpack_small(int bits, const uint8_t *packed, int16_t poly[256]) {
  const int per = 8 / bits;
  for (int i = 0; i < 256; i++) {
    const int code = (packed[i / per] >> ((i % per) * bits)) & ((1 << bits) - 1);
    poly[i] = (int16_t)(code >= (1 << (bits - 1)) ? code - (1 << bits) : code);
  }
}
