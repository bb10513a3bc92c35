// ctx.h -- host-side objects behind the C ABI: RNS rings and IPFE contexts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "cufe_internal.cuh"
#include "prof.h"

namespace cufe {


// An RNS ring Z_q[X]/(X^n + 1) with device twiddle tables.
struct Ring {
  int device = 0, n = 0, logn = 0, k = 0;
  std::vector<uint32_t> q, psi_root;       // primes and the primitive 2n-th roots used
  std::vector<uint32_t> h_psi, h_ipsi;     // host copies [k][n] (bit-reversed powers)
  uint32_t *d_tab = nullptr;               // psi2, ipsi2: 2 x [k][n] (w, w_shoup) pairs
  RingArgs args{};
  int init(int n, int k, const uint32_t *primes, int device);
  void release();
};

// Primes q < 2^31 with q = 1 mod 2^14 (NTT-friendly for every n <= 8192): the params.h
// primes first, then the largest others.
std::vector<uint32_t> ntt_primes(int k);

struct Ctx {
  int device = 0, n = 0, l = 0, num_sms = 148;
  Ring ring;  // k = 3 params.h primes
  cudaStream_t stream = nullptr;
  // scheme constants (src/params.h:14-28 recomputed for this l)
  uint32_t p = 0;
  u128 q = 0, qhalf = 0;
  uint32_t delta_mod[3]{}, delta_sh[3]{};
  uint32_t crt_c1 = 0, crt_c1_sh = 0, crt_c2 = 0, crt_c2_sh = 0;
  // workspace
  uint8_t *ws = nullptr;
  size_t ws_bytes = 0;
  uint32_t *d_status = nullptr;  // sampler status word (device)
  std::mutex mu;                 // serialises host calls on this context
  Prof prof;                     // per-kernel timing (cufe_profile_*)
  // shapes chosen by the tuners (cufe_tune_*): encryption instances per thread group by batch
  // size, coefficient-0 decrypt form by (ciphertexts, keys); absent: the fixed rules
  std::map<int, int> enc_group;
  std::map<std::pair<int, int>, int> coef0_form;
  int enc_group_forced = 0;  // set by the encryption tuner while it times one form

  int init(int n, int l, int device);
  void release();
  int ensure_ws(size_t bytes);
  // NULL selects the legacy default stream, as everywhere in CUDA
  cudaStream_t pick(void *s) const { return static_cast<cudaStream_t>(s); }
  int check_status(cudaStream_t s);  // synchronises s and reports the sampler status word
};

int ntt_launch(const RingArgs &ra, uint32_t *data, long long nres, bool inverse, cudaStream_t s);
int ntt_fwd_shoup_launch(const RingArgs &ra, uint32_t *data, uint32_t *sh, long long nres, cudaStream_t s);
// times the NTT variants on npoly scratch polynomials, keeps the fastest per direction in
// r.args; ms[2 * CUFE_NTT_VARIANTS] (optional): {fwd v1.., inv v1..} in ms per launch
int ring_tune(Ring &r, long long npoly, float *ms, cudaStream_t s);

int ctx_setup_cpu_map(Ctx &c, const uint8_t *seed_a, const uint8_t *seed_s, const uint8_t *seed_e, uint32_t *d_mpk,
                      uint32_t *d_msk, cudaStream_t s);
// setup of one instance of length l (c.l is only the context's default length)
int ctx_setup_cpu_map_l(Ctx &c, int l, const uint8_t *seed_a, const uint8_t *seed_s, const uint8_t *seed_e,
                        uint32_t *d_mpk, uint32_t *d_msk, cudaStream_t s);
int ctx_setup_gpu_map(Ctx &c, const uint8_t *seed2, const uint8_t *seed3, uint32_t *d_mpk, uint32_t *d_msk,
                      cudaStream_t s);
int ctx_encrypt_cpu_map(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                        const uint8_t *seeds3, uint32_t *d_ct, cudaStream_t s);
int ctx_encrypt_gpu_map(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seed2,
                        uint32_t *d_ct, cudaStream_t s);
int ctx_keygen(Ctx &c, int nkeys, const uint32_t *d_y, int y_signed, const uint32_t *d_msk, uint32_t *d_sky,
               cudaStream_t s);
int ctx_decrypt(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                const uint32_t *d_sky, uint32_t *d_dy, cudaStream_t s);
int ctx_decrypt_noalloc(Ctx &c, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                        const uint32_t *d_sky, uint32_t *d_dy, cudaStream_t s);
int ctx_decode(Ctx &c, int count, const uint32_t *d_dy, int ncoeff, uint32_t *d_out, cudaStream_t s);
long long serialized_bytes(const Ctx &c, int kind, int count);
int ctx_serialize(Ctx &c, int kind, int count, const uint32_t *d_src, uint8_t *d_dst, cudaStream_t s);
int ctx_deserialize(Ctx &c, int kind, int count, const uint8_t *d_src, size_t src_bytes, uint32_t *d_dst,
                    cudaStream_t s);
struct SvmModel;
int svm_create(Ctx &c, SvmModel &m, int nr_class, int lsv, const int32_t *sv, int y_signed, const int *nsv,
               const double *sv_coef, const double *rho, const int *label, const uint32_t *d_msk, cudaStream_t s);
int svm_predict(Ctx &c, SvmModel &m, int nct, const uint32_t *d_ct, int *d_label, uint32_t *d_kval, double *d_dec,
                cudaStream_t s);
int svm_tune(Ctx &c, SvmModel &m, int nct, const uint32_t *d_ct, int *choice, float *ms, cudaStream_t s);
SvmModel *svm_new();
void svm_delete(SvmModel *m);
int ctx_decrypt_coef0(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                      const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, cudaStream_t s);
int ctx_decrypt_coef0_form(Ctx &c, int form, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y,
                           int y_signed, const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, cudaStream_t s);
// the tuners: time every form on the caller's buffers (all bit-exact), keep the fastest in c
int ctx_tune_encrypt(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                     const uint8_t *seeds3, uint32_t *d_ct, int *choice, float *ms, cudaStream_t s);
int ctx_tune_decrypt_coef0(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                           const uint32_t *d_sky, uint32_t *d_out, int *choice, float *ms, cudaStream_t s);
int ctx_sample_cpu_map(Ctx &c, int sig, int nstreams, const uint8_t *keys, int calls, uint32_t *d_out,
                       cudaStream_t s);
int ctx_sample_gpu_map(Ctx &c, int sig, const uint8_t *key, int poly0, int npolys, uint32_t *d_out,
                       cudaStream_t s);
int ctx_sample_polya(Ctx &c, const uint8_t *seed, uint32_t *d_a, cudaStream_t s);

}  // namespace cufe
