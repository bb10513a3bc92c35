/*
 * cufe_oracle.c -- CPU restatement of cuFE's RLWE inner-product FE path.
 *
 * TEST INFRASTRUCTURE ONLY (see cufe_oracle.h).  Each function names the reference
 * file:line it restates; paths are relative to the cuFE source tree.
 */
#include "cufe_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

/* ------------------------------------------------------------------ parameters */

/* RNS primes q_j = 2^k1 - 2^k2 + 1 (src/params.h:19, src/arith_rns.c:7-18) */
static const uint32_t OR_Q[3] = {16760833u, 2147352577u, 2130706433u};
static const int OR_K1[3] = {24, 31, 31};
static const int OR_K2[3] = {14, 17, 24};
/* psi_j = primitive 8192-th root of unity used by the reference twiddle tables
 * (src/consts.h: psi[j][k] = psi_j^{bitrev12(k)}, so psi_j = psi[j][2048]). */
static const uint32_t OR_PSI8192[3] = {3689u, 1689795u, 456478u};

struct or_params {
  int n, l, logn;
  uint32_t *psi[3], *psi_inv[3];
  uint32_t ninv[3];
  uint32_t crt_c[3];
  uint32_t p;
  u128 q, delta;
  uint32_t delta_mod[3];
};

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = r * b % q;
    b = b * b % q;
    e >>= 1;
  }
  return r;
}
static uint64_t invmod(uint64_t a, uint64_t q) { return powmod(a, q - 2, q); }

static unsigned bitrev(unsigned x, int bits) {
  unsigned r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

/* primitive 2n-th root consistent with the reference tables (psi_{2n}^{8192/2n} chain) */
static uint32_t root_2n(int j, int n) {
  uint64_t q = OR_Q[j];
  if (2 * n <= 8192) return (uint32_t)powmod(OR_PSI8192[j], 8192 / (2 * n), q);
  /* 2n = 16384: the smaller square root of psi_8192 (all three primes have 2^14 | q-1) */
  uint64_t g = 2;
  for (;; g++) { /* element of order exactly 16384 */
    uint64_t h = powmod(g, (q - 1) / 16384, q);
    if (powmod(h, 8192, q) == q - 1) {
      uint64_t best = 0;
      for (uint64_t t = 1; t < 16384; t += 2) {
        uint64_t c = powmod(h, t, q);
        if (c * c % q == OR_PSI8192[j] && (best == 0 || c < best)) best = c;
      }
      return (uint32_t)best;
    }
  }
}

or_params *or_params_new(int n, int l) {
  if (n < 16 || n > 8192 || (n & (n - 1)) || l < 1) return NULL;
  or_params *P = (or_params *)calloc(1, sizeof(or_params));
  P->n = n;
  P->l = l;
  while ((1 << P->logn) < n) P->logn++;
  for (int j = 0; j < 3; j++) {
    uint64_t q = OR_Q[j], w = root_2n(j, n), wi = invmod(w, q);
    P->psi[j] = (uint32_t *)malloc(sizeof(uint32_t) * n);
    P->psi_inv[j] = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (int k = 0; k < n; k++) {
      unsigned e = bitrev((unsigned)k, P->logn);
      P->psi[j][k] = (uint32_t)powmod(w, e, q);
      P->psi_inv[j][k] = (uint32_t)powmod(wi, e, q);
    }
    P->ninv[j] = (uint32_t)invmod((uint64_t)n, q);
  }
  /* Garner constants (src/params.h:17; the second is stored unreduced there) */
  P->crt_c[0] = 0;
  P->crt_c[1] = (uint32_t)invmod(OR_Q[0], OR_Q[1]);
  P->crt_c[2] = (uint32_t)invmod((uint64_t)OR_Q[0] * OR_Q[1] % OR_Q[2], OR_Q[2]);
  P->p = 4u * 16u * (uint32_t)l + 1u; /* B_x*B_y*l + 1 (src/params.h:26) */
  P->q = (u128)OR_Q[0] * OR_Q[1] * OR_Q[2];
  P->delta = P->q / P->p; /* floor(q/p) (src/params.h:27-28) */
  for (int j = 0; j < 3; j++) P->delta_mod[j] = (uint32_t)(P->delta % OR_Q[j]);
  return P;
}

void or_params_free(or_params *P) {
  if (!P) return;
  for (int j = 0; j < 3; j++) {
    free(P->psi[j]);
    free(P->psi_inv[j]);
  }
  free(P);
}

void or_params_export(const or_params *P, uint32_t *psi, uint32_t *psi_inv, uint32_t *ninv,
                      uint32_t *delta_mod, uint32_t *p_out, uint32_t *q_limbs,
                      uint32_t *delta_limbs) {
  int n = P->n;
  for (int j = 0; j < 3; j++) {
    if (psi) memcpy(psi + j * n, P->psi[j], sizeof(uint32_t) * n);
    if (psi_inv) memcpy(psi_inv + j * n, P->psi_inv[j], sizeof(uint32_t) * n);
    if (ninv) ninv[j] = P->ninv[j];
    if (delta_mod) delta_mod[j] = P->delta_mod[j];
    if (q_limbs) q_limbs[j] = (uint32_t)(P->q >> (32 * j));
    if (delta_limbs) delta_limbs[j] = (uint32_t)(P->delta >> (32 * j));
  }
  if (p_out) *p_out = P->p;
}

/* ------------------------------------------------------------------ arithmetic */

/* src/arith_rns.c:62-83: fold 2^k1 = 2^k2 - 1 while m > 2q, then one conditional
 * subtract.  The result lies in [0, q]; q itself is possible. */
uint32_t or_mod_prime(uint64_t m, int sel) {
  const uint64_t q = OR_Q[sel];
  const int k1 = OR_K1[sel], k2 = OR_K2[sel];
  while (m > 2 * q) m = (m & ((1ull << k1) - 1)) + (((m >> k1) << k2) - (m >> k1));
  if (m >= q) m -= q;
  return (uint32_t)m;
}
/* src/arith_rns.c:23-59 */
static uint32_t add_mod(uint32_t a, uint32_t b, int sel) {
  uint64_t c = (uint64_t)a + b;
  if (c >= OR_Q[sel]) c -= OR_Q[sel];
  return (uint32_t)c;
}
static uint32_t sub_mod(uint32_t a, uint32_t b, int sel) {
  uint64_t c = (uint64_t)a + OR_Q[sel] - b;
  if (c >= OR_Q[sel]) c -= OR_Q[sel];
  return (uint32_t)c;
}
static uint32_t mul_mod(uint32_t a, uint32_t b, int sel) {
  return or_mod_prime((uint64_t)a * b, sel);
}

/* ------------------------------------------------------------------ NTT */

/* src/ntt.c:38-67: Cooley-Tukey, natural order in, bit-reversed order out */
void or_ct_forward(const or_params *P, uint32_t *a, int sel) {
  const int n = P->n;
  int t = n;
  for (int m = 1; m < n; m <<= 1) {
    t >>= 1;
    for (int i = 0; i < m; i++) {
      int j1 = 2 * i * t;
      uint32_t S = P->psi[sel][m + i];
      for (int j = j1; j < j1 + t; j++) {
        uint32_t U = a[j], V = mul_mod(a[j + t], S, sel);
        a[j] = add_mod(U, V, sel);
        a[j + t] = sub_mod(U, V, sel);
      }
    }
  }
}

/* src/ntt.c:70-114: Gentleman-Sande, bit-reversed in, natural out, times n^-1 */
void or_gs_reverse(const or_params *P, uint32_t *a, int sel) {
  const int n = P->n;
  int t = 1;
  for (int m = n; m > 1; m >>= 1) {
    int j1 = 0, h = m / 2;
    for (int i = 0; i < h; i++) {
      uint32_t S = P->psi_inv[sel][h + i];
      for (int j = j1; j < j1 + t; j++) {
        uint32_t U = a[j], V = a[j + t];
        a[j] = add_mod(U, V, sel);
        a[j + t] = mul_mod(sub_mod(U, V, sel), S, sel);
      }
      j1 += 2 * t;
    }
    t <<= 1;
  }
  for (int i = 0; i < n; i++) a[i] = mul_mod(a[i], P->ninv[sel], sel);
}

void or_ntt_generic(uint32_t *a, int n, uint32_t q, const uint32_t *tab, int inverse,
                    uint32_t ninv) {
  if (!inverse) {
    int t = n;
    for (int m = 1; m < n; m <<= 1) {
      t >>= 1;
      for (int i = 0; i < m; i++) {
        uint64_t S = tab[m + i];
        for (int j = 2 * i * t; j < 2 * i * t + t; j++) {
          uint64_t U = a[j], V = (uint64_t)a[j + t] * S % q;
          a[j] = (uint32_t)((U + V) % q);
          a[j + t] = (uint32_t)((U + q - V) % q);
        }
      }
    }
  } else {
    int t = 1;
    for (int m = n; m > 1; m >>= 1) {
      int j1 = 0, h = m / 2;
      for (int i = 0; i < h; i++) {
        uint64_t S = tab[h + i];
        for (int j = j1; j < j1 + t; j++) {
          uint64_t U = a[j], V = a[j + t];
          a[j] = (uint32_t)((U + V) % q);
          a[j + t] = (uint32_t)((U + q - V) % q * S % q);
        }
        j1 += 2 * t;
      }
      t <<= 1;
    }
    for (int i = 0; i < n; i++) a[i] = (uint32_t)((uint64_t)a[i] * ninv % q);
  }
}

/* ------------------------------------------------------------------ AES-256 */
/* FIPS-197.  The S-box is computed from GF(2^8) inversion + affine map. */

static uint8_t SBOX[256];
static uint32_t TE[4][256];
static int aes_ready = 0;

static uint8_t gmul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  while (b) {
    if (b & 1) r ^= a;
    a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
    b >>= 1;
  }
  return r;
}
static void aes_init(void) {
  if (aes_ready) return;
  for (int x = 0; x < 256; x++) {
    uint8_t inv = 0;
    if (x) {
      for (int y = 1; y < 256; y++)
        if (gmul((uint8_t)x, (uint8_t)y) == 1) {
          inv = (uint8_t)y;
          break;
        }
    }
    uint8_t s = inv;
    for (int r = 1; r <= 4; r++) s ^= (uint8_t)((inv << r) | (inv >> (8 - r)));
    SBOX[x] = s ^ 0x63;
  }
  for (int x = 0; x < 256; x++) {
    uint32_t s = SBOX[x];
    uint32_t t = ((uint32_t)gmul((uint8_t)s, 2) << 24) | (s << 16) | (s << 8) | gmul((uint8_t)s, 3);
    TE[0][x] = t;
    TE[1][x] = (t >> 8) | (t << 24);
    TE[2][x] = (t >> 16) | (t << 16);
    TE[3][x] = (t >> 24) | (t << 8);
  }
  aes_ready = 1;
}

static uint32_t be32(const uint8_t *p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}
static void put_be32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)(v >> 24);
  p[1] = (uint8_t)(v >> 16);
  p[2] = (uint8_t)(v >> 8);
  p[3] = (uint8_t)v;
}
static uint64_t le64(const uint8_t *p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
  return v;
}
static uint32_t le32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

void or_aes256_expand(const uint8_t key[32], uint8_t rk[240]) {
  aes_init();
  uint32_t w[60];
  uint8_t rc = 1;
  for (int i = 0; i < 8; i++) w[i] = be32(key + 4 * i);
  for (int i = 8; i < 60; i++) {
    uint32_t t = w[i - 1];
    if (i % 8 == 0) {
      t = (t << 8) | (t >> 24);
      t = ((uint32_t)SBOX[t >> 24] << 24) | ((uint32_t)SBOX[(t >> 16) & 255] << 16) |
          ((uint32_t)SBOX[(t >> 8) & 255] << 8) | SBOX[t & 255];
      t ^= (uint32_t)rc << 24;
      rc = gmul(rc, 2);
    } else if (i % 8 == 4) {
      t = ((uint32_t)SBOX[t >> 24] << 24) | ((uint32_t)SBOX[(t >> 16) & 255] << 16) |
          ((uint32_t)SBOX[(t >> 8) & 255] << 8) | SBOX[t & 255];
    }
    w[i] = w[i - 8] ^ t;
  }
  for (int i = 0; i < 60; i++) put_be32(rk + 4 * i, w[i]);
}

static void aes_words(const uint32_t *w, const uint8_t in[16], uint8_t out[16]) {
  uint32_t s0 = be32(in) ^ w[0], s1 = be32(in + 4) ^ w[1], s2 = be32(in + 8) ^ w[2],
           s3 = be32(in + 12) ^ w[3];
  for (int r = 1; r < 14; r++) {
    const uint32_t *k = w + 4 * r;
    uint32_t t0 = TE[0][s0 >> 24] ^ TE[1][(s1 >> 16) & 255] ^ TE[2][(s2 >> 8) & 255] ^ TE[3][s3 & 255] ^ k[0];
    uint32_t t1 = TE[0][s1 >> 24] ^ TE[1][(s2 >> 16) & 255] ^ TE[2][(s3 >> 8) & 255] ^ TE[3][s0 & 255] ^ k[1];
    uint32_t t2 = TE[0][s2 >> 24] ^ TE[1][(s3 >> 16) & 255] ^ TE[2][(s0 >> 8) & 255] ^ TE[3][s1 & 255] ^ k[2];
    uint32_t t3 = TE[0][s3 >> 24] ^ TE[1][(s0 >> 16) & 255] ^ TE[2][(s1 >> 8) & 255] ^ TE[3][s2 & 255] ^ k[3];
    s0 = t0; s1 = t1; s2 = t2; s3 = t3;
  }
  const uint32_t *k = w + 56;
#define SB(x) ((uint32_t)SBOX[(x)])
  uint32_t o0 = (SB(s0 >> 24) << 24) ^ (SB((s1 >> 16) & 255) << 16) ^ (SB((s2 >> 8) & 255) << 8) ^ SB(s3 & 255) ^ k[0];
  uint32_t o1 = (SB(s1 >> 24) << 24) ^ (SB((s2 >> 16) & 255) << 16) ^ (SB((s3 >> 8) & 255) << 8) ^ SB(s0 & 255) ^ k[1];
  uint32_t o2 = (SB(s2 >> 24) << 24) ^ (SB((s3 >> 16) & 255) << 16) ^ (SB((s0 >> 8) & 255) << 8) ^ SB(s1 & 255) ^ k[2];
  uint32_t o3 = (SB(s3 >> 24) << 24) ^ (SB((s0 >> 16) & 255) << 16) ^ (SB((s1 >> 8) & 255) << 8) ^ SB(s2 & 255) ^ k[3];
#undef SB
  put_be32(out, o0);
  put_be32(out + 4, o1);
  put_be32(out + 8, o2);
  put_be32(out + 12, o3);
}

static void rk_words(const uint8_t rk[240], uint32_t w[60]) {
  for (int i = 0; i < 60; i++) w[i] = be32(rk + 4 * i);
}

void or_aes256_block(const uint8_t rk[240], const uint8_t in[16], uint8_t out[16]) {
  aes_init();
  uint32_t w[60];
  rk_words(rk, w);
  aes_words(w, in, out);
}

/* ------------------------------------------------------------------ CTR stream */
/* src/aes256ctr.c:13-81 (aesni_encrypt8), 83-139 (init), 145-155 (squeeze):
 * block = BE16(nonce) || 0^6 || 0^4 || BE32(ctr + i), 32-bit counter from 0,
 * eight blocks per 128-byte squeeze, counter += 8. */
struct or_ctr {
  uint32_t w[60];
  uint16_t nonce;
  uint32_t ctr;
};

or_ctr *or_ctr_new(const uint8_t *key, uint16_t nonce) {
  aes_init();
  or_ctr *c = (or_ctr *)calloc(1, sizeof(or_ctr));
  if (key) {
    uint8_t rk[240];
    or_aes256_expand(key, rk);
    rk_words(rk, c->w);
  }
  c->nonce = nonce;
  c->ctr = 0;
  return c;
}
void or_ctr_free(or_ctr *c) { free(c); }
uint32_t or_ctr_counter(const or_ctr *c) { return c->ctr; }

void or_ctr_squeeze(or_ctr *c, uint8_t *out, unsigned nblocks128) {
  for (unsigned b = 0; b < nblocks128; b++) {
    for (int i = 0; i < 8; i++) {
      uint8_t in[16] = {0};
      in[0] = (uint8_t)(c->nonce >> 8);
      in[1] = (uint8_t)c->nonce;
      put_be32(in + 12, c->ctr + (uint32_t)i);
      aes_words(c->w, in, out + 16 * i);
    }
    c->ctr += 8;
    out += 128;
  }
}

/* ------------------------------------------------------------------ samplers */

/* binary-sampler scale factors K_i with sigma_i = K_i * sigma_0 (src/gauss.c:11-13) */
static const uint64_t OR_KS[3] = {266ull, 304214978ull, 608429953ull};

/* CDT of the one-sided base sampler D_{sigma_0}^+ as (low63, high63) pairs, entry i =
 * P(x > i) in 126-bit fixed point (src/gauss.c:63-73).  Kept identical: every sample
 * bit depends on it. */
static const uint64_t OR_CDT[9][2] = {
    {2200310400551559144ull, 3327841033070651387ull},
    {7912151619254726620ull, 380075531178589176ull},
    {5167367257772081627ull, 11604843442081400ull},
    {5081592746475748971ull, 90134450315532ull},
    {6522074513864805092ull, 175786317361ull},
    {2579734681240182346ull, 85801740ull},
    {8175784047440310133ull, 10472ull},
    {2947787991558061753ull, 0ull},
    {22489665999543ull, 0ull}};

/* Horner coefficients of the 2^f, f in [0,1), polynomial (src/gauss.c:102-111).
 * Kept identical: the Bernoulli decision compares against its exact double bits. */
static const uint64_t OR_EXPC[10] = {0x3e833b70ffa2c5d4ull, 0x3eb4a480fda7e6e1ull, 0x3ef01b254493363full,
                                     0x3f242e0e0aa273ccull, 0x3f55d8a2334ed31bull, 0x3f83b2aa56db0f1aull,
                                     0x3fac6b08e11fc57eull, 0x3fcebfbdff556072ull, 0x3fe62e42fefa7fe6ull,
                                     0x3ff0000000000000ull};

static double dbits(uint64_t u) {
  double d;
  memcpy(&d, &u, 8);
  return d;
}
static uint64_t ubits(double d) {
  uint64_t u;
  memcpy(&u, &d, 8);
  return u;
}

/* uniform y in [0, K) by 32-bit rejection against K*floor(2^32/K) and Barrett
 * reduction (src/gauss.c:578-703).  Reads consecutive little-endian words from r. */
static int uniform8(int sig, const uint8_t *r, const uint8_t *r_end, uint64_t y[8]) {
  const uint64_t K = OR_KS[sig], BF = (1ull << 32) / K, UQ = K * BF;
  unsigned i = 0;
  for (int j = 0; j < 8; j++) {
    uint64_t x;
    do {
      if (r + 4 * (i + 1) > r_end) return -1; /* beyond the refill buffer: reference UB */
      x = le32(r + 4 * i);
      i++;
    } while (!((x - UQ) >> 63));
    x = x - ((((x * BF) >> 32) + 1) * K);
    x = x + (x >> 63) * K;
    y[j] = x;
  }
  return 0;
}

/* CDT base sample for one lane.  full = 0: high-word compare only, as
 * cdt_sampler64 (src/gauss.c:157-197) and cdt_sampler_gpu (src/sampler.cuh:153-181)
 * compute it (the low-word term is dead).  full = 1: the 126-bit compare of the AVX
 * cdt_sampler (src/gauss.c:122-154) used by the CPU S3. */
static uint64_t cdt_lane(const uint8_t *base, int lane, int full) {
  const uint64_t M = 0x7fffffffffffffffull;
  uint64_t r1 = le64(base + 8 * lane) & M, r2 = le64(base + 32 + 8 * lane) & M, x = 0;
  for (int i = 0; i < 9; i++) {
    uint64_t lt = r2 - OR_CDT[i][1];
    if (full) {
      uint64_t eq = (r2 == OR_CDT[i][1]) ? ~0ull : 0ull;
      lt |= (r1 - OR_CDT[i][0]) & eq;
    }
    x += lt >> 63;
  }
  return x;
}

/* Bernoulli(2^{-x/K^2}) for one lane, returning the word whose bit 63 is the accept bit.
 * Three variants of the same steps, differing only where the reference is undefined:
 *   BV_SCALAR: bernoulli_sampler_S1_64 / S2_64 (src/gauss.c:266-358, 418-520), compiled
 *     x86 code: (int64_t) of an out-of-range double gives INT64_MIN (cvttsd2si) and
 *     `1 << e` masks the count to 6 bits (S2_64 tests e >= 0 first);
 *   BV_AVX: the AVX bernoulli_sampler_S3 (src/gauss.c:524-576) used by the CPU S3:
 *     floor(x) becomes an integer by subtracting double bit patterns, and sllv gives 0
 *     for counts outside [0,63];
 *   BV_GPU: the device functions (src/sampler.cuh:183-422): cvt.rzi.s64.f64 saturates
 *     and PTX shl.b64 clamps (0 outside [0,63]).
 * S1 converts the input with an integer subtract, S2/S3 with the 2^52 bit-cast trick.
 * The Horner chain is fused multiply-add, as the reference builds contract it. */
enum { BV_SCALAR = 0, BV_AVX = 1, BV_GPU = 2 };
static uint64_t bernoulli_lane(int sig, int var, uint64_t xin, const uint8_t *rm, uint8_t rexp) {
  const double K = (double)(int64_t)(OR_KS[sig] * OR_KS[sig]);
  const double kinv = -1.0 / K;
  double vx;
  uint64_t x = xin | 0x4330000000000000ull;
  if (sig == 0)
    vx = (double)(x - 0x4330000000000000ull);
  else
    vx = dbits(x) - 4503599627370496.0;
  vx = vx * kinv;
  double fl = floor(vx);
  double t = fl + 6755399441055744.0;
  uint64_t vtu;
  if (var == BV_AVX) {
    vtu = (ubits(t) - ubits(6755399441055744.0)) << 52;
  } else {
    int64_t ti;
    if (t >= 9223372036854775808.0) ti = (var == BV_GPU) ? INT64_MAX : INT64_MIN;
    else if (t < -9223372036854775808.0) ti = INT64_MIN;
    else ti = (int64_t)t;
    vtu = ((uint64_t)ti - 0x0018000000000000ull) << 52;
  }
  double f = vx - fl;
  double s = fma(dbits(OR_EXPC[0]), f, dbits(OR_EXPC[1]));
  for (int c = 2; c < 10; c++) s = fma(s, f, dbits(OR_EXPC[c]));
  int64_t vres = (int64_t)(vtu + ubits(s));
  int64_t rmant = (vres & ((1ll << 52) - 1)) | (1ll << 52);
  int64_t rexpo;
  if (var == BV_AVX)
    rexpo = (int64_t)((uint64_t)vres >> 52) + (19 - 1023 + 1);
  else
    rexpo = (vres >> 52) + (19 - 1023 + 1);
  int64_t rexp_pow;
  if (var != BV_SCALAR)
    rexp_pow = (rexpo >= 0 && rexpo < 64) ? (int64_t)(1ull << rexpo) : 0;
  else if (sig == 0 || rexpo >= 0)
    rexp_pow = (int64_t)(1ull << (rexpo & 63));
  else
    rexp_pow = 0;
  uint64_t w = le64(rm);
  int64_t r_exp = (int64_t)(((w >> 53) & 0x7ff) | ((uint64_t)rexp << 11));
  int64_t r_mant = (int64_t)(w & ((1ull << 53) - 1));
  uint64_t eq1 = (vres == (1023ll << 52)) ? ~0ull : 0ull;
  return ((uint64_t)(r_mant - rmant) & (uint64_t)(r_exp - rexp_pow)) | eq1;
}

/* mapping 0: the CPU functions (S3 uses the AVX compare and shift); 1: the GPU kernels */
static int candidates(int sig, int mapping, const uint8_t r[384], uint64_t z[8], uint64_t b[8]) {
  const int cdt_full = (mapping == 0 && sig == 2);
  const int var = mapping == 1 ? BV_GPU : (sig == 2 ? BV_AVX : BV_SCALAR);
  uint64_t y[8];
  if (uniform8(sig, r + 200, r + 384, y)) return -1;
  const uint64_t K = OR_KS[sig];
  for (int h = 0; h < 2; h++) {
    const uint8_t *base = r + 100 * h;
    for (int lane = 0; lane < 4; lane++) {
      uint64_t x = cdt_lane(base, lane, cdt_full);
      uint64_t kx = (uint64_t)(uint32_t)x * K;
      uint64_t zz = kx + y[4 * h + lane];
      uint64_t vb = (uint64_t)(uint32_t)(zz + kx) * y[4 * h + lane];
      z[4 * h + lane] = zz;
      b[4 * h + lane] = bernoulli_lane(sig, var, vb, base + 64 + 8 * lane, base[96 + lane]);
    }
  }
  return 0;
}

void or_candidates(int sig, int mapping, const uint8_t r[384], uint64_t z[8], uint64_t b[8]) {
  if (candidates(sig, mapping, r, z, b)) {
    fprintf(stderr, "oracle: uniform sampler ran past the refill buffer\n");
    abort();
  }
}

/* residues of the signed sample (1-2k) z (src/gauss.c:892-904) */
static void emit(uint64_t z, uint64_t k, uint32_t *out, int n, int j) {
  for (int m = 0; m < 3; m++) {
    uint32_t md = or_mod_prime(z, m);
    out[m * n + j] = (uint32_t)((1 - k) * md + k * or_mod_prime(OR_Q[m] - md, m));
  }
}

static int accept(uint64_t b, uint64_t z, uint64_t k) {
  return (int)(((b & ((z | (0 - z)) | (k | (0 - k)))) >> 63) & 1);
}

/* src/gauss.c:789-912 (S1), 995-1084 (S2), 1086-1163 (S3): every call starts with a
 * fresh 384-byte refill (3 squeezes) and drops unused candidates at its end. */
void or_gauss_call(const or_params *P, or_ctr *c, int sig, uint32_t *out, int n) {
  (void)P;
  uint8_t r[384];
  uint64_t z[8], b[8], k;
  unsigned i = 8;
  for (int j = 0; j < n; j++) {
    do {
      if (i == 8) {
        or_ctr_squeeze(c, r, 3);
        or_candidates(sig, 0, r, z, b);
        i = 0;
      }
      k = (r[280] >> i) & 1u;
      i++;
    } while (!accept(b[i - 1], z[i - 1], k));
    emit(z[i - 1], k, out, n, j);
  }
}

/* ------------------------------------------------------------------ GPU counter mapping */

/* src/AES.cuh:380-435: block 0 = AES_K(0^12 || BE32(counter)); block m = AES_K(block_{m-1}
 * XOR K[0:16]) (the round loop restarts from the previous output without a new
 * initial AddRoundKey); 24 blocks per 384-byte refill. */
void or_modeB_refill(const uint8_t rk[240], uint32_t counter, uint8_t out[384]) {
  aes_init();
  uint32_t w[60];
  rk_words(rk, w);
  uint8_t in[16] = {0};
  put_be32(in + 12, counter);
  aes_words(w, in, out);
  for (int m = 1; m < 24; m++) {
    for (int i = 0; i < 16; i++) in[i] = out[16 * (m - 1) + i] ^ rk[i];
    aes_words(w, in, out + 16 * m);
  }
}

/* src/sample_gpu.cu:40-99 / 101-161 / 217-289 with src/AES.cuh:653-665: thread t of
 * polynomial `poly` emits coefficients 8t..8t+7; refill rep uses counter
 * poly*5*T*24 + rep*T*24 + t*24 with T = n/8 threads (T = 512 at n = 4096). */
void or_gauss_modeB_poly(const or_params *P, const uint8_t rk[240], int sig, int poly,
                         uint32_t *out) {
  const int n = P->n, T = n / 8;
  uint8_t r[384];
  uint64_t z[8], b[8], k;
  for (int t = 0; t < T; t++) {
    unsigned i = 8, rep = 0;
    for (int j = 0; j < 8; j++) {
      do {
        if (i == 8) {
          uint32_t ctr = (uint32_t)poly * 5u * (uint32_t)T * 24u + rep * (uint32_t)T * 24u + (uint32_t)t * 24u;
          or_modeB_refill(rk, ctr, r);
          or_candidates(sig, 1, r, z, b);
          i = 0;
          rep++;
        }
        k = (r[280] >> i) & 1u;
        i++;
      } while (!accept(b[i - 1], z[i - 1], k));
      emit(z[i - 1], k, out, n, 8 * t + j);
    }
  }
}

/* ------------------------------------------------------------------ uniform a */

/* src/sample.c:56-128 (active variant: SEC_LEVEL undefined): a_i = le64(buf[8i..]) mod q_j;
 * the comparison against q never rejects a 64-bit value. */
void or_sample_polya(const or_params *P, const uint8_t seed[32], uint32_t *a) {
  const int n = P->n;
  unsigned rounds = (unsigned)(88 * n / 8 / 128);
  uint8_t *buf = (uint8_t *)malloc((size_t)rounds * 128);
  or_ctr *c = or_ctr_new(seed, 0);
  or_ctr_squeeze(c, buf, rounds);
  for (int i = 0; i < n; i++) {
    uint64_t v = le64(buf + 8 * i);
    for (int j = 0; j < 3; j++) a[j * n + i] = (uint32_t)(v % OR_Q[j]);
  }
  or_ctr_free(c);
  free(buf);
}

/* ------------------------------------------------------------------ scheme, CPU mapping */

/* src/rlwe_sife.c:32-82 */
void or_setup(const or_params *P, const uint8_t seed_a[32], const uint8_t *seed_s,
              const uint8_t seed_e[32], uint32_t *mpk, uint32_t *msk) {
  const int n = P->n, l = P->l;
  uint32_t *a = mpk + (size_t)l * 3 * n;
  uint32_t *e = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n);
  uint32_t *t = (uint32_t *)malloc(sizeof(uint32_t) * n);
  or_sample_polya(P, seed_a, a);
  or_ctr *ce = or_ctr_new(seed_e, 0), *cs = or_ctr_new(seed_s, 0);
  for (int j = 0; j < 3; j++) or_ct_forward(P, a + j * n, j);
  for (int i = 0; i < l; i++) {
    uint32_t *s = msk + (size_t)i * 3 * n, *pk = mpk + (size_t)i * 3 * n;
    or_gauss_call(P, cs, 0, s, n);
    or_gauss_call(P, ce, 0, e, n);
    for (int j = 0; j < 3; j++) {
      memcpy(t, s + j * n, sizeof(uint32_t) * n);
      or_ct_forward(P, t, j);
      or_ct_forward(P, e + j * n, j);
      for (int k = 0; k < n; k++) {
        uint32_t v = mul_mod(a[j * n + k], t[k], j);
        pk[j * n + k] = add_mod(v, e[j * n + k], j);
      }
    }
  }
  or_ctr_free(ce);
  or_ctr_free(cs);
  free(e);
  free(t);
}

static void scale_message(const or_params *P, const uint32_t *x, uint32_t *mc) {
  for (int i = 0; i < P->l; i++)
    for (int j = 0; j < 3; j++)
      mc[j * P->l + i] = or_mod_prime((uint64_t)or_mod_prime(x[i], j) * P->delta_mod[j], j);
}

/* src/rlwe_sife.c:112-181 */
void or_encrypt(const or_params *P, const uint32_t *x, const uint32_t *mpk,
                const uint8_t seed2[32], const uint8_t *seed3, uint32_t *ct) {
  const int n = P->n, l = P->l;
  uint32_t *mc = (uint32_t *)malloc(sizeof(uint32_t) * 3 * l);
  uint32_t *r = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n);
  uint32_t *f = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n);
  scale_message(P, x, mc);
  or_ctr *c2 = or_ctr_new(seed2, 0);
  or_gauss_call(P, c2, 1, r, n);
  or_gauss_call(P, c2, 1, f, n);
  for (int j = 0; j < 3; j++) or_ct_forward(P, r + j * n, j);
  for (int j = 0; j < 3; j++) {
    uint32_t *c = ct + ((size_t)l * 3 + j) * n;
    const uint32_t *a = mpk + ((size_t)l * 3 + j) * n;
    for (int k = 0; k < n; k++) c[k] = mul_mod(a[k], r[j * n + k], j);
    or_gs_reverse(P, c, j);
    for (int k = 0; k < n; k++) c[k] = add_mod(c[k], f[j * n + k], j);
  }
  or_ctr *c3 = or_ctr_new(seed3, 0);
  for (int i = 0; i < l; i++) {
    or_gauss_call(P, c3, 2, f, n);
    for (int j = 0; j < 3; j++) {
      uint32_t *c = ct + ((size_t)i * 3 + j) * n;
      const uint32_t *pk = mpk + ((size_t)i * 3 + j) * n;
      for (int k = 0; k < n; k++) c[k] = mul_mod(pk[k], r[j * n + k], j);
      or_gs_reverse(P, c, j);
      for (int k = 0; k < n; k++) {
        c[k] = add_mod(c[k], f[j * n + k], j);
        c[k] = or_mod_prime((uint64_t)(uint32_t)(c[k] + mc[j * l + i]), j);
      }
    }
  }
  or_ctr_free(c2);
  or_ctr_free(c3);
  free(mc);
  free(r);
  free(f);
}

/* src/rlwe_sife.c:215-245 */
void or_keygen(const or_params *P, const uint32_t *y, const uint32_t *msk, uint32_t *sky) {
  const int n = P->n, l = P->l;
  memset(sky, 0, sizeof(uint32_t) * 3 * n);
  for (int i = 0; i < l; i++)
    for (int j = 0; j < 3; j++) {
      uint32_t yc = or_mod_prime(y[i], j);
      const uint32_t *s = msk + ((size_t)i * 3 + j) * n;
      for (int k = 0; k < n; k++)
        sky[j * n + k] = or_mod_prime((uint64_t)yc * s[k] + sky[j * n + k], j);
    }
}

/* src/rlwe_sife.c:248-286 (up to, not including, crt_reverse_gmp) */
void or_decrypt(const or_params *P, const uint32_t *ct, const uint32_t *y,
                const uint32_t *sky, uint32_t *dy) {
  const int n = P->n, l = P->l;
  uint32_t *ta = (uint32_t *)malloc(sizeof(uint32_t) * n);
  uint32_t *tb = (uint32_t *)malloc(sizeof(uint32_t) * n);
  memset(dy, 0, sizeof(uint32_t) * 3 * n);
  for (int i = 0; i < l; i++)
    for (int j = 0; j < 3; j++) {
      uint32_t yc = or_mod_prime(y[i], j);
      const uint32_t *c = ct + ((size_t)i * 3 + j) * n;
      for (int k = 0; k < n; k++)
        dy[j * n + k] = or_mod_prime((uint64_t)yc * c[k] + dy[j * n + k], j);
    }
  for (int j = 0; j < 3; j++) { /* poly_mul_ntt (src/ntt.c:10-26) then poly_sub_mod */
    memcpy(ta, ct + ((size_t)l * 3 + j) * n, sizeof(uint32_t) * n);
    memcpy(tb, sky + (size_t)j * n, sizeof(uint32_t) * n);
    or_ct_forward(P, ta, j);
    or_ct_forward(P, tb, j);
    for (int k = 0; k < n; k++) ta[k] = mul_mod(ta[k], tb[k], j);
    or_gs_reverse(P, ta, j);
    for (int k = 0; k < n; k++) dy[j * n + k] = sub_mod(dy[j * n + k], ta[k], j);
  }
  free(ta);
  free(tb);
}

/* src/crt.c:46-81 (Garner, GMP mod is non-negative) and src/rlwe_sife.c:288-332
 * (quotient of p*x by q, plus one iff the remainder exceeds floor(q/2)). */
void or_decode(const or_params *P, const uint32_t *dy, uint32_t *out, int ncoeff) {
  const int n = P->n;
  const u128 qh = P->q / 2;
  for (int k = 0; k < ncoeff; k++) {
    i128 x = dy[k];
    i128 prod = 1;
    for (int i = 1; i < 3; i++) {
      prod *= OR_Q[i - 1];
      i128 u = ((i128)dy[i * n + k] - x) * (i128)P->crt_c[i];
      u %= (i128)OR_Q[i];
      if (u < 0) u += OR_Q[i];
      x += u * prod;
    }
    u128 a = (u128)x * P->p;
    u128 quo = a / P->q, rem = a % P->q;
    if (rem > qh) quo += 1;
    out[k] = (uint32_t)quo;
  }
}

/* ------------------------------------------------------------------ scheme, GPU mapping */

/* src/rlwe_sife_gpu.cu:19-99 */
void or_setup_modeB(const or_params *P, const uint8_t seed2[32], const uint8_t seed3[32],
                    uint32_t *mpk, uint32_t *msk) {
  const int n = P->n, l = P->l;
  uint8_t rk2[240], rk3[240];
  or_aes256_expand(seed2, rk2);
  or_aes256_expand(seed3, rk3);
  uint32_t *a = mpk + (size_t)l * 3 * n;
  uint32_t *e = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n);
  uint32_t *t = (uint32_t *)malloc(sizeof(uint32_t) * n);
  for (int j = 0; j < 3; j++) or_ct_forward(P, a + j * n, j);
  for (int i = 0; i < l; i++) {
    uint32_t *s = msk + (size_t)i * 3 * n, *pk = mpk + (size_t)i * 3 * n;
    or_gauss_modeB_poly(P, rk2, 0, i, s);
    or_gauss_modeB_poly(P, rk3, 0, i, e);
    for (int j = 0; j < 3; j++) {
      memcpy(t, s + j * n, sizeof(uint32_t) * n);
      or_ct_forward(P, t, j);
      or_ct_forward(P, e + j * n, j);
      for (int k = 0; k < n; k++) pk[j * n + k] = add_mod(mul_mod(a[j * n + k], t[k], j), e[j * n + k], j);
    }
  }
  free(e);
  free(t);
}

/* src/rlwe_sife_gpu.cu:102-188 with the key-buffer overread (Q6) and the 4th-residue
 * write of the S3 kernel (src/sample_gpu.cu:284) resolved: every instance reads the
 * seed2 key; r and f_0 come from the same key and counters, so f_0 == r. */
void or_encrypt_modeB(const or_params *P, const uint32_t *x, const uint32_t *mpk,
                      const uint8_t seed2[32], int repeat, uint32_t *ct) {
  const int n = P->n, l = P->l;
  uint8_t rk[240];
  or_aes256_expand(seed2, rk);
  uint32_t *r = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n);
  uint32_t *f0 = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n);
  uint32_t *f = (uint32_t *)malloc(sizeof(uint32_t) * 3 * n * (size_t)l);
  uint32_t *mc = (uint32_t *)malloc(sizeof(uint32_t) * 3 * l);
  or_gauss_modeB_poly(P, rk, 1, 0, r);
  memcpy(f0, r, sizeof(uint32_t) * 3 * n);
  for (int i = 0; i < l; i++) or_gauss_modeB_poly(P, rk, 2, i, f + (size_t)i * 3 * n);
  for (int j = 0; j < 3; j++) or_ct_forward(P, r + j * n, j);
  for (int rep = 0; rep < repeat; rep++) {
    uint32_t *cr = ct + (size_t)rep * (l + 1) * 3 * n;
    scale_message(P, x + (size_t)rep * l, mc);
    for (int j = 0; j < 3; j++) {
      uint32_t *c = cr + ((size_t)l * 3 + j) * n;
      const uint32_t *a = mpk + ((size_t)l * 3 + j) * n;
      for (int k = 0; k < n; k++) c[k] = mul_mod(r[j * n + k], a[k], j);
      or_gs_reverse(P, c, j);
      for (int k = 0; k < n; k++) c[k] = add_mod(c[k], f0[j * n + k], j);
    }
    for (int i = 0; i < l; i++)
      for (int j = 0; j < 3; j++) {
        uint32_t *c = cr + ((size_t)i * 3 + j) * n;
        const uint32_t *pk = mpk + ((size_t)i * 3 + j) * n;
        for (int k = 0; k < n; k++) c[k] = mul_mod(r[j * n + k], pk[k], j);
        or_gs_reverse(P, c, j);
        for (int k = 0; k < n; k++) {
          c[k] = add_mod(c[k], f[((size_t)i * 3 + j) * n + k], j);
          c[k] = or_mod_prime((uint64_t)(uint32_t)(c[k] + mc[j * l + i]), j);
        }
      }
  }
  free(r);
  free(f0);
  free(f);
  free(mc);
}
