/*
 * cufe_oracle.h -- CPU restatement of cuFE's RLWE inner-product FE path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product in
 * cufe_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it; nothing in the product path links, calls or falls back to it.
 *
 * Parity status: pinned.  The restatement is checked bit-for-bit (canonical residues)
 * against the reference's own CPU sources compiled unmodified (oracle/ref/build_ref.py
 * -> oracle/_ref/) and against the committed fixtures in tests/golden/.
 *
 * Conventions (reference: src/rlwe_sife.h:10-26): polynomial-major layouts
 *   mpk[l+1][3][n], msk[l][3][n], ct[l+1][3][n], sk_y[3][n], d_y[3][n]; x, y uint32[l].
 * Index l of mpk holds NTT(a); index l of ct holds c_0 (the reference's c[SIFE_L]).
 */
#ifndef CUFE_ORACLE_H
#define CUFE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_params or_params;
typedef struct or_ctr or_ctr;

/* parameter set for ring degree n (power of two, 16..8192) and vector length l,
 * with the params.h RNS primes and bounds B_x=4, B_y=16 (p = 64*l + 1). */
or_params *or_params_new(int n, int l);
void or_params_free(or_params *P);
/* table export for tests: psi/psi_inv [3][n], ninv[3], delta_mod[3], p, q limbs (3 x u32) */
void or_params_export(const or_params *P, uint32_t *psi, uint32_t *psi_inv, uint32_t *ninv,
                      uint32_t *delta_mod, uint32_t *p_out, uint32_t *q_limbs, uint32_t *delta_limbs);

/* arithmetic (src/arith_rns.c) */
uint32_t or_mod_prime(uint64_t m, int sel);

/* NTT (src/ntt.c) on one residue polynomial with modulus index sel */
void or_ct_forward(const or_params *P, uint32_t *a, int sel);
void or_gs_reverse(const or_params *P, uint32_t *a, int sel);
/* generic-prime NTT with the same loop structure; psi/psi_inv are bit-reversed power tables */
void or_ntt_generic(uint32_t *a, int n, uint32_t q, const uint32_t *psi_tab, int inverse,
                    uint32_t ninv);

/* AES-256 (FIPS-197) */
void or_aes256_expand(const uint8_t key[32], uint8_t rk[240]);
void or_aes256_block(const uint8_t rk[240], const uint8_t in[16], uint8_t out[16]);

/* AES-256-CTR stream of src/aes256ctr.c.  key == NULL gives the all-zero round-key
 * state that the reference's uninitialised contexts hold when built with
 * -ftrivial-auto-var-init=zero (src/rlwe_sife.c:40 state_secret, :120 state_s3). */
or_ctr *or_ctr_new(const uint8_t *key, uint16_t nonce);
void or_ctr_free(or_ctr *c);
void or_ctr_squeeze(or_ctr *c, uint8_t *out, unsigned nblocks128);
uint32_t or_ctr_counter(const or_ctr *c);

/* one call of gaussian_sampler_S{1,2,3} (src/gauss.c:789,995,1086): n samples into
 * out[3][n] (residues, reference-exact including non-canonical q). sig: 0,1,2. */
void or_gauss_call(const or_params *P, or_ctr *c, int sig, uint32_t *out, int n);

/* refill-level helper for tests: the 8 candidates (z, accept-bit-63 word) the reference
 * derives from one 384-byte refill buffer.  mapping 0: CPU functions, 1: GPU kernels. */
void or_candidates(int sig, int mapping, const uint8_t r[384], uint64_t z[8], uint64_t b[8]);

/* GPU counter mapping (src/AES.cuh:380-435,653-665; src/sample_gpu.cu:40-289).
 * threads = n/8 per polynomial, 8 samples per thread; poly = blockIdx.x. */
void or_modeB_refill(const uint8_t rk[240], uint32_t counter, uint8_t out[384]);
void or_gauss_modeB_poly(const or_params *P, const uint8_t rk[240], int sig, int poly,
                         uint32_t *out);

/* uniform a (src/sample.c:56-128) */
void or_sample_polya(const or_params *P, const uint8_t seed[32], uint32_t *a);

/* scheme, CPU stream mapping (src/rlwe_sife.c).  seed_s / seed3 == NULL selects the
 * zero round-key stream the reference CPU path uses for s_i and f_i. */
void or_setup(const or_params *P, const uint8_t seed_a[32], const uint8_t *seed_s,
              const uint8_t seed_e[32], uint32_t *mpk, uint32_t *msk);
void or_encrypt(const or_params *P, const uint32_t *x, const uint32_t *mpk,
                const uint8_t seed2[32], const uint8_t *seed3, uint32_t *ct);
void or_keygen(const or_params *P, const uint32_t *y, const uint32_t *msk, uint32_t *sky);
void or_decrypt(const or_params *P, const uint32_t *ct, const uint32_t *y,
                const uint32_t *sky, uint32_t *dy);
/* crt_reverse_gmp + round_extract_gmp: d_y residues [3][n] -> integers in [0, p] */
void or_decode(const or_params *P, const uint32_t *dy, uint32_t *out, int ncoeff);

/* scheme, GPU counter mapping (src/rlwe_sife_gpu.cu) with its undefined behaviour
 * resolved: a_coeff is mpk[l] in the coefficient domain on entry. */
void or_setup_modeB(const or_params *P, const uint8_t seed2[32], const uint8_t seed3[32],
                    uint32_t *mpk, uint32_t *msk);
void or_encrypt_modeB(const or_params *P, const uint32_t *x, const uint32_t *mpk,
                      const uint8_t seed2[32], int repeat, uint32_t *ct);

#ifdef __cplusplus
}
#endif
#endif
