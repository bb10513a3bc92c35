// svm.cu -- encrypted linear-SVM prediction (the svm_predict5 path, main.c:270-390).
//
// The reference, per test vector, derives a function key for every support vector
// (rlwe_sife_keygen_gpu with repeat = l SVs), decrypts the test ciphertext under each of
// them (rlwe_sife_decrypt_gmp_gpu), decodes coefficient 0 on the host with GMP
// (round_extract_gmp2, src/rlwe_sife.c:334-393) into kvalue[i] = <x, SV_i>, and takes the
// libsvm one-against-one vote over sv_coef and rho (main.c:331-379).  Here the support
// vectors' function keys are derived once and stay resident; prediction of a batch of
// ciphertexts is the constant-coefficient decryption of every (ciphertext, SV) pair
// followed by the vote, both on the device.
#include <cuda_runtime.h>

#include <vector>

#include "ctx.h"
#include "prof.h"
#include "scheme.cuh"

namespace cufe {

namespace {

constexpr int kMaxClasses = 64;

// One term loop of the vote, `for (k = 0; k < cnt; k++) sum += coef[k] * kvalue[k]`
// (main.c:359-362), with the arithmetic gcc -O3 gives it on an AVX2 + FMA host (the
// reference's Makefile builds with -O3 -march=native -mavx2): the loop is vectorised as an
// in-order reduction, 4 products at a time (vmulpd: each product rounded) added to the sum one
// after another (vaddsd), then a 2-wide epilogue the same way, and an odd last term in the
// scalar remainder, where the multiply-add is contracted to one fused multiply-add.  So every
// product is rounded before its addition except the last one of an odd-length loop.
template <class F>
__device__ double vote_terms(double sum, const double *__restrict__ coef, F value, int first, int cnt) {
  const int paired = cnt & ~1;
  for (int k = 0; k < paired; ++k) sum = __dadd_rn(sum, __dmul_rn(coef[first + k], value(first + k)));
  if (cnt & 1) sum = __fma_rn(coef[first + paired], value(first + paired), sum);
  return sum;
}

// One thread per test vector: the vote of main.c:331-379, in its order, the term loops as
// vote_terms computes them.  kvalue is the decoded coefficient 0 in [0, p]; for signed support
// vectors it is centred into (-p/2, p/2] (the reference only has unsigned y and uses the value
// as decoded).
__global__ void k_svm_vote(const uint32_t *__restrict__ kval, int nct, int lsv, uint32_t p, int centre,
                           int nr_class, const double *__restrict__ coef, const double *__restrict__ rho,
                           const int *__restrict__ nsv, const int *__restrict__ label, int *__restrict__ out,
                           double *__restrict__ dec) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nct) return;
  const uint32_t *kv = kval + (size_t)t * lsv;
  auto value = [&](int i) -> double {
    const uint32_t v = kv[i];
    if (centre) {
      const uint32_t r = v % p;
      return r > p / 2 ? (double)r - (double)p : (double)r;
    }
    return (double)v;
  };
  int start[kMaxClasses], vote[kMaxClasses];
  start[0] = 0;
  for (int i = 1; i < nr_class; ++i) start[i] = start[i - 1] + nsv[i - 1];
  for (int i = 0; i < nr_class; ++i) vote[i] = 0;
  int pp = 0;
  const int npairs = nr_class * (nr_class - 1) / 2;
  for (int i = 0; i < nr_class; ++i)
    for (int j = i + 1; j < nr_class; ++j) {
      double sum = 0;
      const int si = start[i], sj = start[j], ci = nsv[i], cj = nsv[j];
      const double *coef1 = coef + (size_t)(j - 1) * lsv, *coef2 = coef + (size_t)i * lsv;
      sum = vote_terms(sum, coef1, value, si, ci);
      sum = vote_terms(sum, coef2, value, sj, cj);
      sum -= rho[pp];
      if (dec) dec[(size_t)t * npairs + pp] = sum;
      if (sum > 0)
        ++vote[i];
      else
        ++vote[j];
      ++pp;
    }
  int best = 0;
  for (int i = 1; i < nr_class; ++i)
    if (vote[i] > vote[best]) best = i;
  out[t] = label[best];
}

}  // namespace

struct SvmModel {
  int nr_class = 0, lsv = 0, y_signed = 0;
  uint32_t *d_y = nullptr;    // [lsv][l] support vectors (zero beyond their features)
  uint32_t *d_sky = nullptr;  // [lsv][3][n] function keys
  double *d_coef = nullptr, *d_rho = nullptr;
  int *d_nsv = nullptr, *d_label = nullptr;
  uint32_t *d_kval = nullptr;  // [cap][lsv] scratch of predict
  int cap = 0;
  void release() {
    for (void *q : {(void *)d_y, (void *)d_sky, (void *)d_coef, (void *)d_rho, (void *)d_nsv, (void *)d_label,
                    (void *)d_kval})
      if (q) cudaFree(q);
    *this = SvmModel{};
  }
};

SvmModel *svm_new() { return new SvmModel; }
void svm_delete(SvmModel *m) {
  if (m) m->release();
  delete m;
}

int svm_create(Ctx &c, SvmModel &m, int nr_class, int lsv, const int32_t *sv, int y_signed, const int *nsv,
               const double *sv_coef, const double *rho, const int *label, const uint32_t *d_msk, cudaStream_t s) {
  if (nr_class < 2 || nr_class > kMaxClasses || lsv < 1 || !sv || !nsv || !sv_coef || !rho || !label || !d_msk)
    return CUFE_ERR_INVALID;
  long long tot = 0;
  for (int i = 0; i < nr_class; ++i) {
    if (nsv[i] < 0) return CUFE_ERR_INVALID;
    tot += nsv[i];
  }
  if (tot != lsv) {
    set_last_error("svm: nSV must add up to the number of support vectors");
    return CUFE_ERR_INVALID;
  }
  const int npairs = nr_class * (nr_class - 1) / 2;
  m.nr_class = nr_class;
  m.lsv = lsv;
  m.y_signed = y_signed;
  CUFE_CUDA(cudaMalloc(&m.d_y, (size_t)lsv * c.l * 4));
  CUFE_CUDA(cudaMalloc(&m.d_sky, (size_t)lsv * 3 * c.n * 4));
  CUFE_CUDA(cudaMalloc(&m.d_coef, (size_t)(nr_class - 1) * lsv * 8));
  CUFE_CUDA(cudaMalloc(&m.d_rho, (size_t)npairs * 8));
  CUFE_CUDA(cudaMalloc(&m.d_nsv, (size_t)nr_class * 4));
  CUFE_CUDA(cudaMalloc(&m.d_label, (size_t)nr_class * 4));
  CUFE_CUDA(cudaMemcpy(m.d_y, sv, (size_t)lsv * c.l * 4, cudaMemcpyHostToDevice));
  CUFE_CUDA(cudaMemcpy(m.d_coef, sv_coef, (size_t)(nr_class - 1) * lsv * 8, cudaMemcpyHostToDevice));
  CUFE_CUDA(cudaMemcpy(m.d_rho, rho, (size_t)npairs * 8, cudaMemcpyHostToDevice));
  CUFE_CUDA(cudaMemcpy(m.d_nsv, nsv, (size_t)nr_class * 4, cudaMemcpyHostToDevice));
  CUFE_CUDA(cudaMemcpy(m.d_label, label, (size_t)nr_class * 4, cudaMemcpyHostToDevice));
  // the support vectors' function keys, once (rlwe_sife_keygen_gpu with repeat = lsv)
  const int rc = ctx_keygen(c, lsv, m.d_y, y_signed, d_msk, m.d_sky, s);
  if (rc) return rc;
  CUFE_CUDA(cudaStreamSynchronize(s));
  return CUFE_OK;
}

// the model's kvalue scratch for nct test vectors
static int kval_scratch(SvmModel &m, int nct) {
  if (nct > m.cap) {
    if (m.d_kval) CUFE_CUDA(cudaFree(m.d_kval));
    m.d_kval = nullptr;
    CUFE_CUDA(cudaMalloc(&m.d_kval, (size_t)nct * m.lsv * 4));
    m.cap = nct;
  }
  return CUFE_OK;
}

// the coefficient-0 decrypt form for nct test vectors against the model's support vectors
int svm_tune(Ctx &c, SvmModel &m, int nct, const uint32_t *d_ct, int *choice, float *ms, cudaStream_t s) {
  if (nct < 1 || !d_ct) return CUFE_ERR_INVALID;
  const int rc = kval_scratch(m, nct);
  if (rc) return rc;
  return ctx_tune_decrypt_coef0(c, nct, d_ct, m.lsv, m.d_y, m.y_signed, m.d_sky, m.d_kval, choice, ms, s);
}

int svm_predict(Ctx &c, SvmModel &m, int nct, const uint32_t *d_ct, int *d_label, uint32_t *d_kval, double *d_dec,
                cudaStream_t s) {
  if (nct < 1 || !d_ct || !d_label) return CUFE_ERR_INVALID;
  uint32_t *kv = d_kval;
  if (!kv) {
    const int rc = kval_scratch(m, nct);
    if (rc) return rc;
    kv = m.d_kval;
  }
  int rc = ctx_decrypt_coef0(c, nct, d_ct, m.lsv, m.d_y, m.y_signed, m.d_sky, nullptr, kv, s);
  if (rc) return rc;
  ProfScope ps("svm_vote", s);
  note_launch(), k_svm_vote<<<(nct + 127) / 128, 128, 0, s>>>(kv, nct, m.lsv, c.p, m.y_signed, m.nr_class, m.d_coef, m.d_rho,
                                               m.d_nsv, m.d_label, d_label, d_dec);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

}  // namespace cufe
