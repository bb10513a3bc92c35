/*
 * ref_glue.c -- link-time glue for building the reference's CPU path (src/*.c of cuFE,
 * compiled unmodified) into a shared library that tests and the CPU baseline call.
 *
 * TEST INFRASTRUCTURE ONLY.  Provides:
 *   - randombytes(): replaces src/randombytes.c with a queue of caller-chosen 32-byte
 *     seeds, so every randombytes() call of rlwe_sife_setup / rlwe_sife_encrypt
 *     (src/rlwe_sife.c:47,51,139) draws a known seed;
 *   - stubs for the two GPU externs referenced by the *_gui wrappers (src/rlwe_sife.c:23-29),
 *     which the oracle never calls;
 *   - flat ref_* wrappers with plain pointer signatures for ctypes.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <immintrin.h>
#include <gmp.h>

#include "params.h"
#include "aes256ctr.h"
#include "crt.h"
#include "gauss.h"
#include "ntt.h"
#include "rlwe_sife.h"
#include "sample.h"

static unsigned char g_seed_q[256 * 32];
static size_t g_seed_n, g_seed_pos;

void ref_queue_seeds(const unsigned char *seeds, int count) {
  if (count < 0 || count > 256) abort();
  memcpy(g_seed_q, seeds, (size_t)count * 32);
  g_seed_n = (size_t)count * 32;
  g_seed_pos = 0;
}
int ref_seeds_left(void) { return (int)((g_seed_n - g_seed_pos) / 32); }

void randombytes(unsigned char *buf, size_t len) {
  if (g_seed_pos + len > g_seed_n) {
    fprintf(stderr, "ref_glue: randombytes called with no queued seed\n");
    abort();
  }
  memcpy(buf, g_seed_q + g_seed_pos, len);
  g_seed_pos += len;
}

void rlwe_sife_setup_gpu(uint32_t mpk[SIFE_L + 1][SIFE_NMODULI][SIFE_N],
                         uint32_t msk[SIFE_L][SIFE_NMODULI][SIFE_N], unsigned char *seed2,
                         unsigned char *seed3, float *t) {
  (void)mpk; (void)msk; (void)seed2; (void)seed3; (void)t;
  abort();
}
void rlwe_sife_encrypt_gpu(uint32_t *m, uint32_t mpk[SIFE_L + 1][SIFE_NMODULI][SIFE_N],
                           uint32_t *c, unsigned char *seed2, unsigned char *seed3, int repeat,
                           float *t) {
  (void)m; (void)mpk; (void)c; (void)seed2; (void)seed3; (void)repeat; (void)t;
  abort();
}

int ref_n(void) { return SIFE_N; }
int ref_l(void) { return SIFE_L; }

/* setup draws two seeds: a (sample_polya), then the e stream */
void ref_setup(uint32_t *mpk, uint32_t *msk) {
  double t = 0;
  rlwe_sife_setup((uint32_t(*)[SIFE_NMODULI][SIFE_N])mpk, (uint32_t(*)[SIFE_NMODULI][SIFE_N])msk, &t);
}
/* encrypt draws one seed (the S2 stream) */
void ref_encrypt(uint32_t *x, uint32_t *mpk, uint32_t *ct) {
  double t = 0;
  rlwe_sife_encrypt(x, (uint32_t(*)[SIFE_NMODULI][SIFE_N])mpk, (uint32_t(*)[SIFE_NMODULI][SIFE_N])ct, &t);
}
void ref_keygen(const uint32_t *y, const uint32_t *msk, uint32_t *sky) {
  double t = 0;
  rlwe_sife_keygen(y, (const uint32_t(*)[SIFE_NMODULI][SIFE_N])msk, (uint32_t(*)[SIFE_N])sky, &t);
}
/* decrypt + round/extract; writes d_y residues (the GMP CRT value mod q_j) and the
 * decoded integer of every coefficient */
void ref_decrypt(uint32_t *ct, const uint32_t *y, uint32_t *sky, uint32_t *dy_res, uint32_t *decoded) {
  double t = 0;
  mpz_t *dy = (mpz_t *)malloc(sizeof(mpz_t) * SIFE_N);
  for (int i = 0; i < SIFE_N; i++) mpz_init(dy[i]);
  rlwe_sife_decrypt_gmp((uint32_t(*)[SIFE_NMODULI][SIFE_N])ct, y, (uint32_t(*)[SIFE_N])sky, dy, &t);
  for (int j = 0; j < SIFE_NMODULI; j++)
    for (int i = 0; i < SIFE_N; i++) dy_res[j * SIFE_N + i] = (uint32_t)mpz_fdiv_ui(dy[i], SIFE_MOD_Q_I[j]);
  round_extract_gmp(dy);
  for (int i = 0; i < SIFE_N; i++) decoded[i] = (uint32_t)mpz_get_d(dy[i]);
  for (int i = 0; i < SIFE_N; i++) mpz_clear(dy[i]);
  free(dy);
}
/* crt_reverse_gmp + round_extract_gmp on caller residues */
void ref_decode(const uint32_t *res, uint32_t *decoded) {
  mpz_t *a = (mpz_t *)malloc(sizeof(mpz_t) * SIFE_N);
  for (int i = 0; i < SIFE_N; i++) mpz_init(a[i]);
  crt_reverse_gmp(a, (const uint32_t(*)[SIFE_N])res);
  round_extract_gmp(a);
  for (int i = 0; i < SIFE_N; i++) decoded[i] = (uint32_t)mpz_get_d(a[i]);
  for (int i = 0; i < SIFE_N; i++) mpz_clear(a[i]);
  free(a);
}
void ref_ct_forward(uint32_t *a, int sel) { CT_forward(a, (uint32_t)sel); }
void ref_gs_reverse(uint32_t *a, int sel) { GS_reverse(a, (uint32_t)sel); }
void ref_sample_polya(const unsigned char *seed, uint32_t *a) {
  sample_polya((unsigned char *)seed, (uint32_t(*)[SIFE_N])a);
}
/* ncalls consecutive gaussian_sampler_S{sig+1} calls of SIFE_N samples on one stream;
 * key == NULL gives the all-zero context */
void ref_gauss(int sig, const unsigned char *key, int ncalls, uint32_t *out) {
  aes256ctr_ctx *st = (aes256ctr_ctx *)aligned_alloc(32, sizeof(aes256ctr_ctx));
  memset(st, 0, sizeof(*st));
  if (key) aes256ctr_init(st, key, 0);
  for (int c = 0; c < ncalls; c++) {
    uint32_t(*o)[SIFE_N] = (uint32_t(*)[SIFE_N])(out + (size_t)c * SIFE_NMODULI * SIFE_N);
    if (sig == 0) gaussian_sampler_S1(st, o, SIFE_N);
    else if (sig == 1) gaussian_sampler_S2(st, o, SIFE_N);
    else gaussian_sampler_S3(st, o, SIFE_N);
  }
  free(st);
}
/* raw AES-256-CTR stream: nblocks128 squeezes */
void ref_ctr_stream(const unsigned char *key, int nblocks128, unsigned char *out) {
  aes256ctr_ctx *st = (aes256ctr_ctx *)aligned_alloc(32, sizeof(aes256ctr_ctx));
  memset(st, 0, sizeof(*st));
  if (key) aes256ctr_init(st, key, 0);
  aes256ctr_squeezeblocks(out, (unsigned long long)nblocks128, st);
  free(st);
}
