/*
 * cufe_b200.h -- C ABI of cufe_b200, a B200-native (sm_100a) implementation of cuFE's
 * RLWE inner-product functional-encryption path.
 *
 * Two layers:
 *   1. Drop-in symbols with the exact names and argument lists of the reference's GPU
 *      entry points (cuFE src/rlwe_sife_gpu.cu, PERF build), bound by the reference's own
 *      callers (src/rlwe_sife.c:23-29 and main.c:22-28).  Host buffers, synchronous,
 *      reference layouts and the reference GPU counter-to-sample mapping.
 *   2. A context API with runtime ring degree n and vector length l, device pointers and
 *      stream ordering, covering both randomness mappings (the reference CPU path's streams,
 *      bit-exact with svm_predict3, and the GPU kernels' counter mapping), batched
 *      encryption, multi-key keygen, cross-product decryption and on-device decode.
 *
 * Layouts (src/rlwe_sife.h:10-26): mpk[l+1][3][n] with NTT(a) at index l, msk[l][3][n],
 * ct[l+1][3][n] with c_0 at index l, sk_y[3][n], d_y[3][n], x and y uint32[l]; all residues
 * are canonical in [0, q_j).  The three RNS primes are those of src/params.h:19.
 */
#ifndef CUFE_B200_H
#define CUFE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference returns void and checks nothing) */
#define CUFE_OK 0
#define CUFE_ERR_INVALID (-1)     /* bad argument or unsupported size */
#define CUFE_ERR_CUDA (-2)        /* CUDA runtime error; text in cufe_last_error() */
#define CUFE_ERR_NOMEM (-3)       /* device allocation failed */
#define CUFE_ERR_SAMPLER (-4)     /* sampler status word set; outputs of that call are invalid */
#define CUFE_ERR_NODEVICE (-5)    /* no CUDA device */

/* sampler index: sigma_1 (setup), sigma_2 (r, f_0), sigma_3 (f_i) (src/gauss.c:11-13) */
#define CUFE_SIGMA1 0
#define CUFE_SIGMA2 1
#define CUFE_SIGMA3 2

const char *cufe_last_error(void);
const char *cufe_version(void);

/* =====================================================================================
 * 1. Reference drop-in.  Dimensions: those set by cufe_dropin_configure (default n = 4096,
 *    l = 785, the values of src/params.h:21-22).  Failures leave outputs untouched, print
 *    one line to stderr and are reported by cufe_dropin_status().
 * ===================================================================================== */

/* replaces rlwe_sife_setup_gpu (src/rlwe_sife_gpu.cu:19); mpk[l] holds a (coefficient domain)
 * on entry; s_i from seed2, e_i from seed3, GPU counter mapping */
void rlwe_sife_setup_gpu(uint32_t *mpk, uint32_t *msk, unsigned char *seed2, unsigned char *seed3,
                         float *part2_time);
/* replaces rlwe_sife_encrypt_gpu (src/rlwe_sife_gpu.cu:102); m[repeat][l], c[repeat][l+1][3][n];
 * every instance draws r, f_0 and f_i from seed2 as the reference kernels do (seed3 unused) */
void rlwe_sife_encrypt_gpu(uint32_t *m, uint32_t *mpk, uint32_t *c, unsigned char *seed2,
                           unsigned char *seed3, int repeat, float *part2_time);
/* replaces rlwe_sife_keygen_gpu (src/rlwe_sife_gpu.cu:191); y[repeat][l] -> sk_y[repeat][3][n] */
void rlwe_sife_keygen_gpu(const uint32_t *y, const uint32_t *msk, uint32_t *sk_y, int repeat,
                          float *part2_time);
/* replaces rlwe_sife_decrypt_gmp_gpu (src/rlwe_sife_gpu.cu:231); one ciphertext, repeat keys
 * -> d_y[repeat][3][n] residues (undecoded, as the reference) */
void rlwe_sife_decrypt_gmp_gpu(uint32_t *c, const uint32_t *y, uint32_t *sk_y, uint32_t *d_y, int repeat,
                               float *part2_time);

int cufe_dropin_configure(int n, int l, int device);
int cufe_dropin_status(void);

/* =====================================================================================
 * 2. Context API.  Every call is asynchronous and ordered on the `stream` argument
 *    (a cudaStream_t; NULL is the legacy default stream).  Seeds and keys are host pointers
 *    and are consumed before the call returns.
 * ===================================================================================== */

typedef struct cufe_ctx cufe_ctx;

/* n: power of two in [16, 8192]; l: vector length (p = 64 l + 1, Delta = floor(q/p)) */
int cufe_create(cufe_ctx **ctx, int n, int l, int device);
int cufe_destroy(cufe_ctx *ctx);
/* waits for all work queued on `stream` and reports the sampler
 * status word (CUFE_ERR_SAMPLER if any sampler call since the last check hit an undefined
 * reference case or ran out of precomputed refills) */
int cufe_sync(cufe_ctx *ctx, void *stream);
/* a non-blocking stream owned by the context */
void *cufe_ctx_stream(cufe_ctx *ctx);
/* per-kernel device timing: when enabled, every named group of launches (one kernel, or a
 * few for a sampler stage) is bracketed by CUDA events on its stream; cufe_profile_read
 * waits for them and returns, per group name (64-byte slots), the kernels launched in it and
 * the summed milliseconds; returns the number of groups written (or a negative status) */
int cufe_profile_enable(cufe_ctx *ctx, int on);
int cufe_profile_read(cufe_ctx *ctx, int max_kernels, char *names, long long *launches, double *ms);
int cufe_profile_reset(cufe_ctx *ctx);
/* kernel launches of this context's calls while profiling was on, since the last reset (every
 * kernel, inside a named group or not).  No counterpart in the reference. */
long long cufe_profile_launches(const cufe_ctx *ctx);
/* p and floor(q/p) mod q_j */
int cufe_params(const cufe_ctx *ctx, uint32_t *p, uint32_t delta_mod[3]);
/* twiddle tables [3][n] (psi^{bitrev(i)}, psi^{-bitrev(i)}) in host memory */
int cufe_tables(const cufe_ctx *ctx, uint32_t *psi, uint32_t *psi_inv);

/* setup, CPU mapping (rlwe_sife_setup, src/rlwe_sife.c:32-82): a from seed_a
 * (sample_polya), s_i from the seed_s stream (NULL: the all-zero round-key stream of the
 * reference CPU path), e_i from the seed_e stream.  Seeds are host pointers. */
int cufe_setup(cufe_ctx *ctx, const uint8_t seed_a[32], const uint8_t *seed_s, const uint8_t seed_e[32],
               uint32_t *d_mpk, uint32_t *d_msk, void *stream);
/* setup, GPU counter mapping (rlwe_sife_setup_gpu): d_mpk[l] holds a on entry */
int cufe_setup_gpu_map(cufe_ctx *ctx, const uint8_t seed2[32], const uint8_t seed3[32], uint32_t *d_mpk,
                       uint32_t *d_msk, void *stream);

/* batch independent encryptions, CPU mapping (rlwe_sife_encrypt, src/rlwe_sife.c:112-181):
 * instance b draws r and f_0 from seeds2[b], f_i from seeds3[b] (seeds3 NULL: the zero-key
 * stream of the reference CPU path).  d_x[batch][l], d_ct[batch][l+1][3][n]. */
int cufe_encrypt(cufe_ctx *ctx, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                 const uint8_t *seeds3, uint32_t *d_ct, void *stream);
/* GPU counter mapping (rlwe_sife_encrypt_gpu): all instances share seed2's randomness */
int cufe_encrypt_gpu_map(cufe_ctx *ctx, int batch, const uint32_t *d_x, const uint32_t *d_mpk,
                         const uint8_t seed2[32], uint32_t *d_ct, void *stream);

/* sk_y = sum_i y_i msk_i (rlwe_sife_keygen, src/rlwe_sife.c:215-245) for nkeys vectors
 * d_y[nkeys][l]; y_signed = 0 reduces y as uint32 (the reference), 1 as int32 */
int cufe_keygen(cufe_ctx *ctx, int nkeys, const uint32_t *d_y, int y_signed, const uint32_t *d_msk,
                uint32_t *d_sky, void *stream);
/* d_y = sum_i y_i c_i - c_l * sk_y (rlwe_sife_decrypt_gmp before the CRT,
 * src/rlwe_sife.c:248-278) for every (ciphertext, key) pair: d_dy[nct][nkeys][3][n] */
int cufe_decrypt(cufe_ctx *ctx, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                 const uint32_t *d_sky, uint32_t *d_dy, void *stream);
/* Decryption that allocates no device memory, for callers that cannot call cudaMalloc
 * during a call (a host application with a fixed GPU memory budget, or a serving thread
 * that must not take cudaMalloc's implicit device synchronisation).  No counterpart in the
 * reference.  Same result as cufe_decrypt for one ciphertext d_ct[l+1][3][n] and nkeys
 * keys: d_dy[nkeys][3][n].  Limits: n <= 4096 and 1 <= nkeys <= 4, else CUFE_ERR_INVALID.
 * Its scratch is a fixed array of about 2 MiB inside the library image, held on every GPU
 * that loads the library until the process exits.  The first call on a device looks up the
 * array's device address (make that first call before any stream capture).  All calls share
 * the array: calls that overlap on the GPU (different streams, threads or contexts without
 * ordering between them) race and corrupt each other's results. */
int cufe_decrypt_noalloc(cufe_ctx *ctx, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                         const uint32_t *d_sky, uint32_t *d_dy, void *stream);
/* crt_reverse_gmp + round_extract_gmp (src/crt.c:46-81, src/rlwe_sife.c:288-332) on the first
 * ncoeff coefficients of each of count d_y: d_out[count][ncoeff], values in [0, p] */
int cufe_decode(cufe_ctx *ctx, int count, const uint32_t *d_dy, int ncoeff, uint32_t *d_out, void *stream);
/* Decrypt and decode coefficient 0 only, the one coefficient the reference reads after
 * decryption (src/rlwe_sife.c:380; main.c:205, 326).  For every (ciphertext, key) pair:
 * d_out[nct][nkeys] = decode of d_y[0], where d_y[0] = sum_i y_i c_i[0] - (c_l * sk_y)[0] with
 * the negacyclic constant term (c_l * sk_y)[0] = c_l[0] sk_y[0] - sum_{t>=1} c_l[t] sk_y[n-t].
 * Equal to cufe_decode(cufe_decrypt(...), ncoeff = 1).  d_d0 (optional, may be NULL) receives
 * the residues d_d0[nct][nkeys][3]. */
int cufe_decrypt_coef0(cufe_ctx *ctx, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                       const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, void *stream);

/* Shape tuners (no counterpart in the reference, which has one fixed launch shape per kernel).
 * Each times every form of one operation on the caller's buffers -- all forms give the same
 * bits, so the outputs are valid whichever ran last -- and keeps the fastest on the context
 * for that shape; later calls of the same shape use it (other shapes keep the fixed rules).
 *   cufe_tune_encrypt: one or two instances per thread group in the encryption kernel, for this
 *     batch size (fixed rule: two from batch 2); choice = 1 or 2, ms[2];
 *   cufe_tune_decrypt_coef0: for (nct, nkeys), form 0 = one CTA per (ciphertext, key) pair, 1..4
 *     = the tiled product at 64x32, 64x64, 32x32, 32x64 ciphertexts x keys per CTA (fixed rule:
 *     form 0 below 32 keys, else 1); choice = the form, ms[5];
 *   cufe_decrypt_coef0_form: cufe_decrypt_coef0 in the given form (tests, comparisons). */
int cufe_tune_encrypt(cufe_ctx *ctx, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                      const uint8_t *seeds3, uint32_t *d_ct, int *choice, float *ms, void *stream);
int cufe_tune_decrypt_coef0(cufe_ctx *ctx, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                            const uint32_t *d_sky, uint32_t *d_out, int *choice, float *ms, void *stream);
int cufe_decrypt_coef0_form(cufe_ctx *ctx, int form, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y,
                            int y_signed, const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, void *stream);

/* samplers, for parity tests and statistics.  CPU mapping: nstreams AES-CTR streams keyed by
 * keys[nstreams][32] (NULL: zero-key streams), each running `calls` consecutive
 * gaussian_sampler_S* calls of n samples (src/gauss.c:789,995,1086): d_out[nstreams][calls][3][n]. */
int cufe_sample_cpu_map(cufe_ctx *ctx, int sig, int nstreams, const uint8_t *keys, int calls, uint32_t *d_out,
                        void *stream);
/* refills (384-byte AES-CTR blocks of 8 candidates) that the CPU-mapping sampler
 * precomputes per stream for `calls` calls of n samples (sizing and roofline accounting) */
long long cufe_sampler_refills(int sig, int calls, int n);
/* GPU counter mapping (src/sample_gpu.cu:40-289) for polynomials poly0..poly0+npolys-1 */
int cufe_sample_gpu_map(cufe_ctx *ctx, int sig, const uint8_t key[32], int poly0, int npolys, uint32_t *d_out,
                        void *stream);
/* sample_polya (src/sample.c:56-128): d_a[3][n] */
int cufe_sample_polya(cufe_ctx *ctx, const uint8_t seed[32], uint32_t *d_a, void *stream);

/* How the CPU-mapping samplers find where each gaussian_sampler_S* call starts (process-wide;
 * all give the same samples): 0 (default) the cheaper of pointer doubling (parallel over
 * refills, log2(calls) table levels; runs up to 32 Mi refills) and the serial one-warp walk
 * (dependent loads per call of the longest stream), by a cost model measured on a B200;
 * 1 always the walk; 2 doubling whenever the run is within 32 Mi refills.  Applies to
 * workspaces sized after the call. */
int cufe_sampler_call_search(int mode);

/* Serialized keys and ciphertexts: a 32-byte header (magic "CUFE", version 1, kind, n, l,
 * count, residue polynomials per object, payload bytes) and the canonical residues packed at
 * their moduli's bit widths (24, 31, 31 bits; each polynomial padded to 32 bits): 10.75 bytes
 * per coefficient triple instead of 12.  Device buffers, 4-byte aligned; the bytes can be
 * copied to the host and written out as they are.  No counterpart in the reference, which
 * keeps keys and ciphertexts only as C arrays in memory. */
#define CUFE_OBJ_MPK 1 /* [count][l+1][3][n] */
#define CUFE_OBJ_MSK 2 /* [count][l][3][n] */
#define CUFE_OBJ_CT 3  /* [count][l+1][3][n] */
#define CUFE_OBJ_SKY 4 /* [count][3][n] */
#define CUFE_OBJ_DY 5  /* [count][3][n] */
long long cufe_serialized_bytes(const cufe_ctx *ctx, int kind, int count);
/* synchronous on stream */
int cufe_serialize(cufe_ctx *ctx, int kind, int count, const uint32_t *d_src, uint8_t *d_dst, void *stream);
/* synchronous; CUFE_ERR_INVALID if the header does not match (kind, the context's n and l,
 * count) or a residue is not below its modulus */
int cufe_deserialize(cufe_ctx *ctx, int kind, int count, const uint8_t *d_src, size_t src_bytes, uint32_t *d_dst,
                     void *stream);

/* =====================================================================================
 * 2a. Encrypted linear-SVM prediction: the svm_predict5 path (svm_predict_gpu,
 *     main.c:270-390) with the support vectors' function keys derived once and resident.
 * ===================================================================================== */

typedef struct cufe_svm cufe_svm;

/* A libsvm one-against-one model (svm/svm.h:52-72) on the context's parameters: nr_class
 * classes, nsv_total support vectors sv[nsv_total][l] (convertToarray's dense layout,
 * main.c:30-41: feature index -> value, zero elsewhere; sv_signed = 1 allows negative
 * integer entries, 0 is the reference's uint32), nSV[nr_class], sv_coef[nr_class-1][nsv_total],
 * rho[nr_class*(nr_class-1)/2], label[nr_class]; d_msk the master secret key.  Derives the
 * function key of every support vector once (rlwe_sife_keygen, src/rlwe_sife.c:215-245);
 * synchronous. */
int cufe_svm_create(cufe_svm **svm, cufe_ctx *ctx, int nr_class, int nsv_total, const int32_t *sv, int sv_signed,
                    const int *nsv, const double *sv_coef, const double *rho, const int *label, const uint32_t *d_msk,
                    void *stream);
/* Predict nct encrypted test vectors d_ct[nct][l+1][3][n]: kvalue = decoded coefficient 0
 * of every (ciphertext, support vector) decryption, then the vote of main.c:331-379 with
 * fused multiply-adds in the reference's order.  d_label[nct] (device); d_kvalue
 * [nct][nsv_total] and d_dec [nct][pairs] are optional (device, NULL to skip). */
int cufe_svm_predict(cufe_svm *svm, int nct, const uint32_t *d_ct, int *d_label, uint32_t *d_kvalue, double *d_dec,
                     void *stream);
/* the coefficient-0 decrypt form for nct ciphertexts against the model's support vectors
 * (cufe_tune_decrypt_coef0 on the model's keys); choice and ms[5] as there */
int cufe_svm_tune(cufe_svm *svm, int nct, const uint32_t *d_ct, int *choice, float *ms, void *stream);
int cufe_svm_destroy(cufe_svm *svm);

/* =====================================================================================
 * 2b. Heterogeneous batches: many independent instances, each with its own ring degree n_i,
 *     vector length l_i (hence its own p_i = 64 l_i + 1 and floor(q / p_i), src/params.h:26-27)
 *     and master key pair.  No counterpart in the reference, which runs one instance of
 *     compile-time size per process; every step below is the reference's algorithm per
 *     instance (setup src/rlwe_sife.c:32-82, encrypt 112-181, keygen 215-245, decrypt and
 *     decode of coefficient 0 248-332, CPU stream mapping for all randomness).
 * ===================================================================================== */

typedef struct cufe_batch cufe_batch;

/* count instances, n[i] a power of two in [256, 8192], l[i] in [1, 4096].  Keys of all
 * instances stay resident (sum of (2 l_i + 1) * 3 * n_i words); a step processes instances in
 * chunks whose scratch stays below max_chunk_bytes (0: 24 GiB). */
int cufe_batch_create(cufe_batch **batch, int count, const int *n, const int *l, size_t max_chunk_bytes, int device);
int cufe_batch_destroy(cufe_batch *batch);
/* master keys of every instance from host seeds [count][32] (seeds_s may be NULL: the
 * reference's zero-key secret stream) */
int cufe_batch_setup(cufe_batch *batch, const uint8_t *seeds_a, const uint8_t *seeds_s, const uint8_t *seeds_e,
                     void *stream);
/* device buffers of a step: d_x (uint32) and d_y (int32, signed) packed by instance, instance i
 * at word x_off[i] (cufe_batch_info); d_seeds2 / d_seeds3 [count][32] encryption seeds;
 * d_out[count] the decoded coefficient 0 of d_y in [0, p_i] (the inner product mod p_i);
 * d_d0 (optional) [count][3] its residues.  Rebinding different buffers drops the graph. */
int cufe_batch_bind(cufe_batch *batch, const uint32_t *d_x, const int32_t *d_y, const uint8_t *d_seeds2,
                    const uint8_t *d_seeds3, uint32_t *d_out, uint32_t *d_d0);
/* one step with the bound buffers, eagerly on `stream` */
int cufe_batch_run(cufe_batch *batch, void *stream);
/* the same step from a CUDA graph, captured on the first call (after one eager step, made by
 * that call if none ran) and replayed afterwards: the graph reads the bound buffers' current
 * contents, so new seeds or inputs written there take effect on the next replay */
int cufe_batch_replay(cufe_batch *batch, void *stream);
/* Re-lays the chunks of a bound batch for each scratch budget budgets[0..ncand-1] (keys stay
 * resident), times one eager step each and keeps the fastest layout; ms[i] = -1 for a budget
 * whose scratch does not fit the device.  No counterpart in the reference.  Drops the graph. */
int cufe_batch_tune(cufe_batch *batch, int ncand, const size_t *budgets, size_t *chosen, float *ms, void *stream);
/* kernel timing of eager steps (cufe_batch_run): on != 0 clears and starts it; read gives the
 * summed device milliseconds of the step's kernel groups (CUDA events around each group on the
 * step's stream) and the number of kernels launched; with it the cost of the graph's launch
 * gaps is replay time / kernel time.  No counterpart in the reference. */
int cufe_batch_profile(cufe_batch *batch, int on);
int cufe_batch_profile_read(cufe_batch *batch, double *kernel_ms, long long *kernels);
/* the same per named kernel group (64-byte name slots), as cufe_profile_read; returns the
 * number of groups written */
int cufe_batch_profile_groups(cufe_batch *batch, int max_groups, char *names, long long *launches, double *ms);
/* kernel nodes of the captured step graph (0 before the first replay) */
int cufe_batch_graph_kernels(cufe_batch *batch);
/* synchronous check of the batch's sampler status word (CUFE_ERR_SAMPLER if set) */
int cufe_batch_status(cufe_batch *batch);
/* x_off[count + 1] (may be NULL), number of chunks, resident key bytes, scratch bytes */
int cufe_batch_info(const cufe_batch *batch, uint64_t *x_off, int *chunks, size_t *key_bytes, size_t *scratch_bytes);
/* device addresses of instance i's mpk [(l+1)][3][n], msk [l][3][n], function key [3][n] of
 * the last step, and (one-chunk batches after a step, else NULL) its ciphertext [(l+1)][3][n] */
int cufe_batch_instance(const cufe_batch *batch, int i, const uint32_t **mpk, const uint32_t **msk,
                        const uint32_t **sky, const uint32_t **ct);

/* =====================================================================================
 * 2c. Request server over resident tenants (continuous batching).  No counterpart in the
 *     reference.  Tenants are instances with their own (n, l) and key pair (set up as in
 *     section 2b).  Requests are queued on submission and served in ticks: cufe_server_poll
 *     retires finished ticks and launches the next one over every queued request that fits
 *     (arrival order; admission by device-memory footprint: tick scratch, ciphertext arena,
 *     function-key arena), with up to two ticks in flight.  Each request computes the
 *     reference's algorithm on its own inputs only, so its result does not depend on what it
 *     was batched with.  Calls on one server are serialised by a lock.
 * ===================================================================================== */

typedef struct cufe_server cufe_server;

/* tenants with n[i] a power of two in [256, 8192] and l[i] in [1, 4096]; arena_bytes for
 * resident ciphertexts (function keys get a quarter of that), tick_bytes of scratch per tick
 * (0: 16 GiB each) */
int cufe_server_create(cufe_server **server, int tenants, const int *n, const int *l, size_t arena_bytes,
                       size_t tick_bytes, int device);
int cufe_server_destroy(cufe_server *server);
/* tenant key pairs from host seeds [tenants][32] (seeds_s may be NULL); synchronous */
int cufe_server_setup(cufe_server *server, const uint8_t *seeds_a, const uint8_t *seeds_s, const uint8_t *seeds_e);
/* the server's clock in seconds (steady); request arrival times use it */
double cufe_server_now(void);
/* submit a request; host inputs are copied; t_arrival < 0 means now.  Returns a request id
 * (>= 0) or a negative status.  encrypt: x[l] of the tenant, two 32-byte seeds (CPU stream
 * mapping); keygen: signed y[l]; decrypt: a ciphertext and a function key (request ids of
 * the same tenant), result = the decoded coefficient 0 of d_y in [0, p] */
long long cufe_server_encrypt(cufe_server *server, int tenant, const uint32_t *x, const uint8_t *seed2,
                              const uint8_t *seed3, double t_arrival);
long long cufe_server_keygen(cufe_server *server, int tenant, const int32_t *y, double t_arrival);
long long cufe_server_decrypt(cufe_server *server, long long ciphertext, long long function_key, double t_arrival);
/* retire finished ticks and launch the next; wait != 0 first blocks on the oldest tick in
 * flight.  Returns the number of requests completed by this call or a negative status. */
int cufe_server_poll(cufe_server *server, int wait);
int cufe_server_pending(cufe_server *server, long long *queued, int *ticks_in_flight);
/* state: 0 queued, 1 running, 2 done, 3 released, 4 shed (dropped unrun by the overload
 * limits below; no result); value: a decrypt's result */
int cufe_server_result(cufe_server *server, long long id, int *state, uint32_t *value, double *t_arrival,
                       double *t_done);
/* copy a finished encrypt's ciphertext [(l+1)][3][n] or keygen's function key [3][n] (then
 * y[l]) to host memory (synchronous) */
int cufe_server_read(cufe_server *server, long long id, uint32_t *host, size_t words);
/* free a finished encrypt's or keygen's slot once no queued decrypt reads it */
int cufe_server_release(cufe_server *server, long long id);
int cufe_server_stats(cufe_server *server, long long *ticks, long long *done, size_t *ct_free_bytes);
/* Overload control.  A tick admits at most max_tick_requests requests (0: only the memory
 * limits), which bounds how long one tick runs; a queued request that has waited longer than
 * max_queue_seconds (0: no limit) when a tick is formed is shed instead of run (state 4), and so
 * is a decrypt that reads a shed encrypt or keygen.  A completed request's latency is then at
 * most max_queue_seconds plus the time of the tick before it and its own.  Applies from the next
 * tick on. */
int cufe_server_limits(cufe_server *server, int max_tick_requests, double max_queue_seconds);
/* requests shed so far (or a negative status) */
long long cufe_server_shed(cufe_server *server);

/* =====================================================================================
 * 3. Negacyclic NTT on an RNS ring (CT_forward / GS_reverse, src/ntt.c:38-114)
 * ===================================================================================== */

typedef struct cufe_ring cufe_ring;

/* k primes (NULL: the params.h primes, then the largest primes below 2^31 that are 1 mod
 * 2^14); n power of two in [16, 8192], k in [1, 6] */
int cufe_ring_create(cufe_ring **ring, int n, int k, const uint32_t *primes, int device);
int cufe_ring_destroy(cufe_ring *ring);
/* primes[k], roots[k] (the primitive 2n-th roots used), tables [k][n] */
int cufe_ring_info(const cufe_ring *ring, uint32_t *primes, uint32_t *roots, uint32_t *psi, uint32_t *psi_inv);
/* in place on d_data[npoly][k][n]; forward: natural -> bit-reversed order */
int cufe_ntt_forward(const cufe_ring *ring, uint32_t *d_data, long long npoly, void *stream);
int cufe_ntt_inverse(const cufe_ring *ring, uint32_t *d_data, long long npoly, void *stream);
/* Kernel variants and their tuner.  Variant 1: one residue polynomial per thread group,
 * one group per residue, 16 coefficients per thread (radix-16 passes).  Variant 2: two
 * residues of the same modulus (rows 2t and 2t+1) per group, sharing twiddle loads and
 * shared-memory addresses.  Variant 3: persistent groups (a grid of one wave) that load
 * their next residue into registers while transforming the current one.  Variant 4:
 * variant 1 compiled for 5 CTAs per SM (48 registers per thread; 256-thread CTAs).
 * Variants 5 and 6: variant 2 compiled for 3 or 4 CTAs per SM of 256 threads (n = 8192,
 * 512-thread CTAs: 1 or 2).  Variants 7 and 8 (n >= 1024):
 * 32 coefficients per thread (radix-32 passes: n = 1024 in 2 passes, 8192 in 3), compiled
 * for 2 or 3 CTAs per SM.  Variant 9 (n >= 2048): 64 coefficients per thread (radix 64:
 * n = 2048 and 4096 in 2 passes).  On smaller rings variants 7-9 run variant 1.
 * cufe_ring_tune times the CUFE_NTT_VARIANTS variants in both directions on a scratch buffer
 * of npoly polynomials (capped at 1 GiB, allocated and freed inside the call, synchronous)
 * and keeps the fastest per direction; ms (optional, 2 * CUFE_NTT_VARIANTS floats) receives
 * {fwd v1..v9, inv v1..v9} in milliseconds per launch.  A new ring uses variant 6, the
 * fastest form at every n when measured on a B200.  Every variant splits a launch into one
 * grid over the moduli below 2^27 (lazy butterflies: no reduction in the forward until its
 * last stage, [0, 2q) in the inverse) and one over the others.
 * No counterpart in the reference. */
#define CUFE_NTT_VARIANTS 9
int cufe_ring_tune(cufe_ring *ring, long long npoly, float *ms, void *stream);
int cufe_ring_set_variant(cufe_ring *ring, int fwd, int inv);
int cufe_ring_get_variant(const cufe_ring *ring, int *fwd, int *inv);

#ifdef __cplusplus
}
#endif
#endif
