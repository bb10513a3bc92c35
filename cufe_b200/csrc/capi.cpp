// capi.cpp -- extern "C" entry points declared in include/cufe_b200.h.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "ctx.h"
#include "sampler_host.h"
#include "staging.h"

namespace cufe {
thread_local Prof *t_prof = nullptr;
thread_local long long t_launches = 0;
static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace cufe

struct cufe_ctx {
  cufe::Ctx c;
};
struct cufe_ring {
  cufe::Ring r;
};

using cufe::Ctx;

extern "C" {

const char *cufe_last_error(void) { return cufe::g_last_error.c_str(); }
const char *cufe_version(void) { return "cufe_b200 0.1 (sm_100a)"; }

// ------------------------------------------------------------------ context API

static int need_device(int device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    cufe::set_last_error("no CUDA device");
    return CUFE_ERR_NODEVICE;
  }
  if (device < 0 || device >= count) {
    cufe::set_last_error("device index out of range");
    return CUFE_ERR_INVALID;
  }
  return CUFE_OK;
}

static bool pow2_in(int n, int lo, int hi) { return n >= lo && n <= hi && (n & (n - 1)) == 0; }

int cufe_create(cufe_ctx **out, int n, int l, int device) {
  if (!out) return CUFE_ERR_INVALID;
  *out = nullptr;
  if (!pow2_in(n, 16, 8192) || l < 1 || l > 65536) {
    cufe::set_last_error("n must be a power of two in [16, 8192] and l in [1, 65536]");
    return CUFE_ERR_INVALID;
  }
  int rc = need_device(device);
  if (rc) return rc;
  cufe_ctx *h = new (std::nothrow) cufe_ctx();
  if (!h) return CUFE_ERR_NOMEM;
  rc = h->c.init(n, l, device);
  if (rc) {
    h->c.release();
    delete h;
    return rc;
  }
  *out = h;
  return CUFE_OK;
}

int cufe_destroy(cufe_ctx *h) {
  if (!h) return CUFE_ERR_INVALID;
  cudaSetDevice(h->c.device);
  cudaStreamSynchronize(h->c.stream);
  h->c.release();
  delete h;
  return CUFE_OK;
}

void *cufe_ctx_stream(cufe_ctx *h) { return h ? (void *)h->c.stream : nullptr; }

struct ProfBind {
  explicit ProfBind(cufe::Prof *p) { cufe::t_prof = p; }
  ~ProfBind() { cufe::t_prof = nullptr; }
};

#define CTX_CALL(h, expr)                        \
  do {                                           \
    if (!(h)) return CUFE_ERR_INVALID;           \
    std::lock_guard<std::mutex> lk((h)->c.mu);   \
    ProfBind pb(&(h)->c.prof);                   \
    if (cudaSetDevice((h)->c.device) != cudaSuccess) return CUFE_ERR_CUDA; \
    return (expr);                               \
  } while (0)

int cufe_sync(cufe_ctx *h, void *stream) { CTX_CALL(h, h->c.check_status(h->c.pick(stream))); }

int cufe_profile_enable(cufe_ctx *h, int on) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> lk(h->c.mu);
  h->c.prof.collect();
  h->c.prof.on = on != 0;
  return CUFE_OK;
}

int cufe_profile_read(cufe_ctx *h, int max_kernels, char *names, long long *launches, double *ms) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> lk(h->c.mu);
  h->c.prof.collect();
  int i = 0;
  for (auto &kv : h->c.prof.acc) {
    if (i >= max_kernels) break;
    if (names) {
      std::strncpy(names + 64 * (size_t)i, kv.first.c_str(), 63);
      names[64 * (size_t)i + 63] = 0;
    }
    if (launches) launches[i] = kv.second.first;
    if (ms) ms[i] = kv.second.second;
    ++i;
  }
  return i;
}

int cufe_profile_reset(cufe_ctx *h) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> lk(h->c.mu);
  h->c.prof.collect();
  h->c.prof.acc.clear();
  h->c.prof.kernels = 0;
  return CUFE_OK;
}

long long cufe_profile_launches(const cufe_ctx *h) {
  if (!h) return CUFE_ERR_INVALID;
  return h->c.prof.kernels;
}

long long cufe_sampler_refills(int sig, int calls, int n) {
  if (sig < 0 || sig > 2 || calls < 1 || n < 16) return -1;
  return (long long)cufe::cpu_map_refills((uint32_t)calls, (uint32_t)n, sig);
}

int cufe_params(const cufe_ctx *h, uint32_t *p, uint32_t delta_mod[3]) {
  if (!h) return CUFE_ERR_INVALID;
  if (p) *p = h->c.p;
  if (delta_mod)
    for (int j = 0; j < 3; ++j) delta_mod[j] = h->c.delta_mod[j];
  return CUFE_OK;
}

int cufe_tables(const cufe_ctx *h, uint32_t *psi, uint32_t *psi_inv) {
  if (!h) return CUFE_ERR_INVALID;
  const size_t sz = h->c.ring.h_psi.size() * 4;
  if (psi) std::memcpy(psi, h->c.ring.h_psi.data(), sz);
  if (psi_inv) std::memcpy(psi_inv, h->c.ring.h_ipsi.data(), sz);
  return CUFE_OK;
}

int cufe_setup(cufe_ctx *h, const uint8_t seed_a[32], const uint8_t *seed_s, const uint8_t seed_e[32],
               uint32_t *d_mpk, uint32_t *d_msk, void *stream) {
  if (!seed_a || !seed_e || !d_mpk || !d_msk) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_setup_cpu_map(h->c, seed_a, seed_s, seed_e, d_mpk, d_msk, h->c.pick(stream)));
}

int cufe_setup_gpu_map(cufe_ctx *h, const uint8_t seed2[32], const uint8_t seed3[32], uint32_t *d_mpk,
                       uint32_t *d_msk, void *stream) {
  if (!seed2 || !seed3 || !d_mpk || !d_msk) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_setup_gpu_map(h->c, seed2, seed3, d_mpk, d_msk, h->c.pick(stream)));
}

int cufe_encrypt(cufe_ctx *h, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                 const uint8_t *seeds3, uint32_t *d_ct, void *stream) {
  if (!d_x || !d_mpk || !d_ct) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_encrypt_cpu_map(h->c, batch, d_x, d_mpk, seeds2, seeds3, d_ct, h->c.pick(stream)));
}

int cufe_encrypt_gpu_map(cufe_ctx *h, int batch, const uint32_t *d_x, const uint32_t *d_mpk,
                         const uint8_t seed2[32], uint32_t *d_ct, void *stream) {
  if (!d_x || !d_mpk || !d_ct) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_encrypt_gpu_map(h->c, batch, d_x, d_mpk, seed2, d_ct, h->c.pick(stream)));
}

int cufe_keygen(cufe_ctx *h, int nkeys, const uint32_t *d_y, int y_signed, const uint32_t *d_msk,
                uint32_t *d_sky, void *stream) {
  if (!d_y || !d_msk || !d_sky) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_keygen(h->c, nkeys, d_y, y_signed, d_msk, d_sky, h->c.pick(stream)));
}

int cufe_decrypt(cufe_ctx *h, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                 const uint32_t *d_sky, uint32_t *d_dy, void *stream) {
  if (!d_ct || !d_y || !d_sky || !d_dy) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_decrypt(h->c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d_dy, h->c.pick(stream)));
}

int cufe_decrypt_noalloc(cufe_ctx *h, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                         const uint32_t *d_sky, uint32_t *d_dy, void *stream) {
  if (!d_ct || !d_y || !d_sky || !d_dy) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_decrypt_noalloc(h->c, d_ct, nkeys, d_y, y_signed, d_sky, d_dy, h->c.pick(stream)));
}

int cufe_decrypt_coef0(cufe_ctx *h, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                       const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, void *stream) {
  if (!d_ct || !d_y || !d_sky || !d_out) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_decrypt_coef0(h->c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d_d0, d_out, h->c.pick(stream)));
}

int cufe_decrypt_coef0_form(cufe_ctx *h, int form, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y,
                            int y_signed, const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, void *stream) {
  if (!d_ct || !d_y || !d_sky || !d_out) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_decrypt_coef0_form(h->c, form, nct, d_ct, nkeys, d_y, y_signed, d_sky, d_d0, d_out,
                                           h->c.pick(stream)));
}

int cufe_tune_decrypt_coef0(cufe_ctx *h, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                            const uint32_t *d_sky, uint32_t *d_out, int *choice, float *ms, void *stream) {
  if (!d_ct || !d_y || !d_sky || !d_out) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_tune_decrypt_coef0(h->c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d_out, choice, ms,
                                           h->c.pick(stream)));
}

int cufe_tune_encrypt(cufe_ctx *h, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                      const uint8_t *seeds3, uint32_t *d_ct, int *choice, float *ms, void *stream) {
  if (!d_x || !d_mpk || !seeds2 || !d_ct) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_tune_encrypt(h->c, batch, d_x, d_mpk, seeds2, seeds3, d_ct, choice, ms, h->c.pick(stream)));
}

int cufe_decode(cufe_ctx *h, int count, const uint32_t *d_dy, int ncoeff, uint32_t *d_out, void *stream) {
  if (!d_dy || !d_out) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_decode(h->c, count, d_dy, ncoeff, d_out, h->c.pick(stream)));
}

int cufe_sample_cpu_map(cufe_ctx *h, int sig, int nstreams, const uint8_t *keys, int calls, uint32_t *d_out,
                        void *stream) {
  if (!d_out) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_sample_cpu_map(h->c, sig, nstreams, keys, calls, d_out, h->c.pick(stream)));
}

int cufe_sample_gpu_map(cufe_ctx *h, int sig, const uint8_t key[32], int poly0, int npolys, uint32_t *d_out,
                        void *stream) {
  if (!d_out) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_sample_gpu_map(h->c, sig, key, poly0, npolys, d_out, h->c.pick(stream)));
}

int cufe_sample_polya(cufe_ctx *h, const uint8_t seed[32], uint32_t *d_a, void *stream) {
  if (!d_a) return CUFE_ERR_INVALID;
  CTX_CALL(h, cufe::ctx_sample_polya(h->c, seed, d_a, h->c.pick(stream)));
}

// ------------------------------------------------------------------ rings

int cufe_ring_create(cufe_ring **out, int n, int k, const uint32_t *primes, int device) {
  if (!out) return CUFE_ERR_INVALID;
  *out = nullptr;
  if (!pow2_in(n, 16, 8192) || k < 1 || k > cufe::kMaxModuli) {
    cufe::set_last_error("n must be a power of two in [16, 8192] and k in [1, 6]");
    return CUFE_ERR_INVALID;
  }
  if (primes)
    for (int m = 0; m < k; ++m)
      if (primes[m] >= (1u << 31) || (primes[m] - 1) % (2u * (uint32_t)n) != 0) {
        cufe::set_last_error("primes must be below 2^31 and 1 mod 2n");
        return CUFE_ERR_INVALID;
      }
  int rc = need_device(device);
  if (rc) return rc;
  cufe_ring *h = new (std::nothrow) cufe_ring();
  if (!h) return CUFE_ERR_NOMEM;
  rc = h->r.init(n, k, primes, device);
  if (rc) {
    h->r.release();
    delete h;
    return rc;
  }
  *out = h;
  return CUFE_OK;
}

int cufe_ring_destroy(cufe_ring *h) {
  if (!h) return CUFE_ERR_INVALID;
  h->r.release();
  delete h;
  return CUFE_OK;
}

int cufe_ring_info(const cufe_ring *h, uint32_t *primes, uint32_t *roots, uint32_t *psi, uint32_t *psi_inv) {
  if (!h) return CUFE_ERR_INVALID;
  for (int m = 0; m < h->r.k; ++m) {
    if (primes) primes[m] = h->r.q[m];
    if (roots) roots[m] = h->r.psi_root[m];
  }
  const size_t sz = h->r.h_psi.size() * 4;
  if (psi) std::memcpy(psi, h->r.h_psi.data(), sz);
  if (psi_inv) std::memcpy(psi_inv, h->r.h_ipsi.data(), sz);
  return CUFE_OK;
}

int cufe_ntt_forward(const cufe_ring *h, uint32_t *d_data, long long npoly, void *stream) {
  if (!h || !d_data || npoly < 0) return CUFE_ERR_INVALID;
  if (cudaSetDevice(h->r.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return cufe::ntt_launch(h->r.args, d_data, npoly * h->r.k, false, static_cast<cudaStream_t>(stream));
}

int cufe_ntt_inverse(const cufe_ring *h, uint32_t *d_data, long long npoly, void *stream) {
  if (!h || !d_data || npoly < 0) return CUFE_ERR_INVALID;
  if (cudaSetDevice(h->r.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return cufe::ntt_launch(h->r.args, d_data, npoly * h->r.k, true, static_cast<cudaStream_t>(stream));
}

int cufe_ring_tune(cufe_ring *h, long long npoly, float *ms, void *stream) {
  if (!h || npoly < 1) return CUFE_ERR_INVALID;
  if (cudaSetDevice(h->r.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return cufe::ring_tune(h->r, npoly, ms, static_cast<cudaStream_t>(stream));
}

int cufe_ring_set_variant(cufe_ring *h, int fwd, int inv) {
  if (!h || fwd < 1 || fwd > CUFE_NTT_VARIANTS || inv < 1 || inv > CUFE_NTT_VARIANTS) return CUFE_ERR_INVALID;
  h->r.args.pp_fwd = fwd;
  h->r.args.pp_inv = inv;
  return CUFE_OK;
}

int cufe_ring_get_variant(const cufe_ring *h, int *fwd, int *inv) {
  if (!h) return CUFE_ERR_INVALID;
  if (fwd) *fwd = h->r.args.pp_fwd;
  if (inv) *inv = h->r.args.pp_inv;
  return CUFE_OK;
}

long long cufe_serialized_bytes(const cufe_ctx *h, int kind, int count) {
  if (!h) return CUFE_ERR_INVALID;
  return cufe::serialized_bytes(h->c, kind, count);
}

int cufe_serialize(cufe_ctx *h, int kind, int count, const uint32_t *d_src, uint8_t *d_dst, void *stream) {
  CTX_CALL(h, cufe::ctx_serialize(h->c, kind, count, d_src, d_dst, h->c.pick(stream)));
}

int cufe_deserialize(cufe_ctx *h, int kind, int count, const uint8_t *d_src, size_t src_bytes, uint32_t *d_dst,
                     void *stream) {
  CTX_CALL(h, cufe::ctx_deserialize(h->c, kind, count, d_src, src_bytes, d_dst, h->c.pick(stream)));
}

int cufe_sampler_call_search(int mode) {
  if (mode < 0 || mode > 2) return CUFE_ERR_INVALID;
  cufe::set_call_search(mode);
  return CUFE_OK;
}

// ------------------------------------------------------------------ encrypted SVM prediction

struct cufe_svm {
  cufe_ctx *ctx = nullptr;
  cufe::SvmModel *m = nullptr;
};

int cufe_svm_create(cufe_svm **out, cufe_ctx *h, int nr_class, int nsv_total, const int32_t *sv, int sv_signed,
                    const int *nsv, const double *sv_coef, const double *rho, const int *label, const uint32_t *d_msk,
                    void *stream) {
  if (!out || !h) return CUFE_ERR_INVALID;
  *out = nullptr;
  cufe_svm *sm = new cufe_svm;
  sm->ctx = h;
  sm->m = cufe::svm_new();
  int rc;
  {
    std::lock_guard<std::mutex> lk(h->c.mu);
    ProfBind pb(&h->c.prof);
    if (cudaSetDevice(h->c.device) != cudaSuccess) {
      rc = CUFE_ERR_CUDA;
    } else {
      rc = cufe::svm_create(h->c, *sm->m, nr_class, nsv_total, sv, sv_signed, nsv, sv_coef, rho, label, d_msk,
                            h->c.pick(stream));
    }
  }
  if (rc) {
    cufe::svm_delete(sm->m);
    delete sm;
    return rc;
  }
  *out = sm;
  return CUFE_OK;
}

int cufe_svm_predict(cufe_svm *sm, int nct, const uint32_t *d_ct, int *d_label, uint32_t *d_kvalue, double *d_dec,
                     void *stream) {
  if (!sm) return CUFE_ERR_INVALID;
  cufe_ctx *h = sm->ctx;
  CTX_CALL(h, cufe::svm_predict(h->c, *sm->m, nct, d_ct, d_label, d_kvalue, d_dec, h->c.pick(stream)));
}

int cufe_svm_tune(cufe_svm *sm, int nct, const uint32_t *d_ct, int *choice, float *ms, void *stream) {
  if (!sm || !d_ct) return CUFE_ERR_INVALID;
  cufe_ctx *h = sm->ctx;
  CTX_CALL(h, cufe::svm_tune(h->c, *sm->m, nct, d_ct, choice, ms, h->c.pick(stream)));
}

int cufe_svm_destroy(cufe_svm *sm) {
  if (!sm) return CUFE_ERR_INVALID;
  cudaSetDevice(sm->ctx->c.device);
  cufe::svm_delete(sm->m);
  delete sm;
  return CUFE_OK;
}

// ------------------------------------------------------------------ reference drop-in

namespace {
struct Dropin {
  std::mutex mu;
  int n = 4096, l = 785, device = 0;  // src/params.h:21-22
  cufe_ctx *ctx = nullptr;
  int status = CUFE_OK;
  uint32_t *buf = nullptr;
  size_t buf_words = 0;
  cufe::Staging stage;  // the caller's pageable buffers <-> device, through pinned slots
};
Dropin &dropin() {
  static Dropin d;
  return d;
}

int dropin_ready(Dropin &d) {
  if (d.ctx) return CUFE_OK;
  return cufe_create(&d.ctx, d.n, d.l, d.device);
}

int dropin_buf(Dropin &d, size_t words) {
  if (words <= d.buf_words) return CUFE_OK;
  if (d.buf) cudaFree(d.buf);
  d.buf = nullptr;
  d.buf_words = 0;
  if (cudaMalloc(&d.buf, words * 4) != cudaSuccess) {
    cudaGetLastError();
    cufe::set_last_error("drop-in buffer allocation failed");
    return CUFE_ERR_NOMEM;
  }
  d.buf_words = words;
  return CUFE_OK;
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  float *out;
  explicit Timer(float *o) : out(o) {
    if (out) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, 0);
    }
  }
  void done() {
    if (!out) return;
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    *out += ms;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    out = nullptr;
  }
  ~Timer() { done(); }
};

void dropin_fail(Dropin &d, const char *op, int rc) {
  d.status = rc;
  std::fprintf(stderr, "cufe_b200: %s failed (%d): %s\n", op, rc, cufe_last_error());
}

#define DI_CHECK(expr)                     \
  do {                                     \
    int _rc = (expr);                      \
    if (_rc) {                             \
      dropin_fail(d, __func__, _rc);       \
      return;                              \
    }                                      \
  } while (0)
#define DI_CUDA(expr)                                                      \
  do {                                                                     \
    cudaError_t _e = (expr);                                               \
    if (_e != cudaSuccess) {                                               \
      cufe::set_last_error(cudaGetErrorString(_e));                        \
      dropin_fail(d, __func__, CUFE_ERR_CUDA);                             \
      return;                                                              \
    }                                                                      \
  } while (0)
}  // namespace

int cufe_dropin_configure(int n, int l, int device) {
  Dropin &d = dropin();
  std::lock_guard<std::mutex> lk(d.mu);
  if (d.ctx) cufe_destroy(d.ctx);
  d.ctx = nullptr;
  if (d.buf) cudaFree(d.buf);
  d.buf = nullptr;
  d.buf_words = 0;
  d.n = n;
  d.l = l;
  d.device = device;
  d.status = CUFE_OK;
  return dropin_ready(d);
}

int cufe_dropin_status(void) { return dropin().status; }

void rlwe_sife_setup_gpu(uint32_t *mpk, uint32_t *msk, unsigned char *seed2, unsigned char *seed3,
                         float *part2_time) {
  Dropin &d = dropin();
  std::lock_guard<std::mutex> lk(d.mu);
  d.status = CUFE_OK;
  DI_CHECK(dropin_ready(d));
  cudaSetDevice(d.device);
  const size_t poly = (size_t)3 * d.n, L = (size_t)d.l;
  Timer tm(part2_time);
  DI_CHECK(dropin_buf(d, (2 * L + 1) * poly));
  uint32_t *dm = d.buf, *ds = d.buf + (L + 1) * poly;
  DI_CUDA(cudaMemcpy(dm + L * poly, mpk + L * poly, poly * 4, cudaMemcpyHostToDevice));
  DI_CHECK(cufe_setup_gpu_map(d.ctx, seed2, seed3, dm, ds, nullptr));
  DI_CHECK(cufe_sync(d.ctx, nullptr));
  DI_CUDA(d.stage.d2h(mpk, dm, (L + 1) * poly * 4, nullptr));
  DI_CUDA(d.stage.d2h(msk, ds, L * poly * 4, nullptr));
}

void rlwe_sife_encrypt_gpu(uint32_t *m, uint32_t *mpk, uint32_t *c, unsigned char *seed2, unsigned char *seed3,
                           int repeat, float *part2_time) {
  (void)seed3;
  Dropin &d = dropin();
  std::lock_guard<std::mutex> lk(d.mu);
  d.status = CUFE_OK;
  if (repeat < 1) {
    cufe::set_last_error("repeat < 1");
    dropin_fail(d, __func__, CUFE_ERR_INVALID);
    return;
  }
  DI_CHECK(dropin_ready(d));
  cudaSetDevice(d.device);
  const size_t poly = (size_t)3 * d.n, L = (size_t)d.l, R = (size_t)repeat;
  Timer tm(part2_time);
  DI_CHECK(dropin_buf(d, (L + 1) * poly * (1 + R) + R * L));
  uint32_t *dm = d.buf, *dc = d.buf + (L + 1) * poly, *dx = dc + R * (L + 1) * poly;
  DI_CUDA(d.stage.h2d(dm, mpk, (L + 1) * poly * 4, nullptr));
  DI_CUDA(cudaMemcpy(dx, m, R * L * 4, cudaMemcpyHostToDevice));
  DI_CHECK(cufe_encrypt_gpu_map(d.ctx, repeat, dx, dm, seed2, dc, nullptr));
  DI_CHECK(cufe_sync(d.ctx, nullptr));
  DI_CUDA(d.stage.d2h(c, dc, R * (L + 1) * poly * 4, nullptr));
}

void rlwe_sife_keygen_gpu(const uint32_t *y, const uint32_t *msk, uint32_t *sk_y, int repeat, float *part2_time) {
  Dropin &d = dropin();
  std::lock_guard<std::mutex> lk(d.mu);
  d.status = CUFE_OK;
  if (repeat < 1) {
    cufe::set_last_error("repeat < 1");
    dropin_fail(d, __func__, CUFE_ERR_INVALID);
    return;
  }
  DI_CHECK(dropin_ready(d));
  cudaSetDevice(d.device);
  const size_t poly = (size_t)3 * d.n, L = (size_t)d.l, R = (size_t)repeat;
  Timer tm(part2_time);
  DI_CHECK(dropin_buf(d, L * poly + R * poly + R * L));
  uint32_t *ds = d.buf, *dk = ds + L * poly, *dy = dk + R * poly;
  DI_CUDA(d.stage.h2d(ds, msk, L * poly * 4, nullptr));
  DI_CUDA(cudaMemcpy(dy, y, R * L * 4, cudaMemcpyHostToDevice));
  DI_CHECK(cufe_keygen(d.ctx, repeat, dy, 0, ds, dk, nullptr));
  DI_CHECK(cufe_sync(d.ctx, nullptr));
  DI_CUDA(d.stage.d2h(sk_y, dk, R * poly * 4, nullptr));
}

void rlwe_sife_decrypt_gmp_gpu(uint32_t *c, const uint32_t *y, uint32_t *sk_y, uint32_t *d_y, int repeat,
                               float *part2_time) {
  Dropin &d = dropin();
  std::lock_guard<std::mutex> lk(d.mu);
  d.status = CUFE_OK;
  if (repeat < 1) {
    cufe::set_last_error("repeat < 1");
    dropin_fail(d, __func__, CUFE_ERR_INVALID);
    return;
  }
  DI_CHECK(dropin_ready(d));
  cudaSetDevice(d.device);
  const size_t poly = (size_t)3 * d.n, L = (size_t)d.l, R = (size_t)repeat;
  Timer tm(part2_time);
  DI_CHECK(dropin_buf(d, (L + 1) * poly + 2 * R * poly + R * L));
  uint32_t *dc = d.buf, *dk = dc + (L + 1) * poly, *dd = dk + R * poly, *dy = dd + R * poly;
  DI_CUDA(d.stage.h2d(dc, c, (L + 1) * poly * 4, nullptr));
  DI_CUDA(cudaMemcpy(dy, y, R * L * 4, cudaMemcpyHostToDevice));
  DI_CUDA(d.stage.h2d(dk, sk_y, R * poly * 4, nullptr));
  DI_CHECK(cufe_decrypt(d.ctx, 1, dc, repeat, dy, 0, dk, dd, nullptr));
  DI_CHECK(cufe_sync(d.ctx, nullptr));
  DI_CUDA(d.stage.d2h(d_y, dd, R * poly * 4, nullptr));
}

}  // extern "C"
