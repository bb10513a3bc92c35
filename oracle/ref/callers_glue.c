/*
 * callers_glue.c -- link-time glue for oracle/_ref/callers/libcallers.so: the reference's own
 * callers of the GPU entry points (cuFE main.c with main renamed, src/rlwe_sife.c and the rest
 * of src/*.c, svm/svm.cpp), compiled unmodified and linked against libcufe_b200.so, which
 * provides rlwe_sife_{setup,encrypt,keygen}_gpu and rlwe_sife_decrypt_gmp_gpu.
 *
 * TEST INFRASTRUCTURE ONLY.  Provides:
 *   - randombytes(): a queue of caller-chosen 32-byte seeds in place of src/randombytes.c;
 *   - __wrap_malloc / __wrap_free (the library links with --wrap=malloc,--wrap=free): when
 *     armed, two chosen allocations (by their order after arming) are copied out when they
 *     are freed.  svm_predict_cpu allocates dec_values first and kvalue second (main.c:141,
 *     158), svm_predict_gpu dec_values first and kvalue fifth (main.c:276-282), and both free
 *     them at their end, so this reads the decision values and the decoded inner products the
 *     reference computes without touching its source;
 *   - flat cl_* wrappers with plain pointer signatures for ctypes.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "params.h"
#include "rlwe_sife.h"
#include "svm/svm.h"

/* ---------------------------------------------------------------- seeds */
static unsigned char g_seed_q[1024 * 32];
static size_t g_seed_n, g_seed_pos;

void cl_queue_seeds(const unsigned char *seeds, int count) {
  if (count < 0 || count > 1024) abort();
  memcpy(g_seed_q, seeds, (size_t)count * 32);
  g_seed_n = (size_t)count * 32;
  g_seed_pos = 0;
}

void randombytes(unsigned char *buf, size_t len) {
  if (g_seed_pos + len > g_seed_n) {
    fprintf(stderr, "callers_glue: randombytes called with no queued seed\n");
    abort();
  }
  memcpy(buf, g_seed_q + g_seed_pos, len);
  g_seed_pos += len;
}

/* ---------------------------------------------------------------- allocation capture */
void *__real_malloc(size_t n);
void __real_free(void *p);

static int g_armed, g_count;         /* capturing; allocations seen since arming */
static int g_index[2];               /* which allocations (0-based, after arming) to keep */
static void *g_ptr[2];
static size_t g_bytes[2];
static unsigned char g_copy[2][65536];

void *__wrap_malloc(size_t n) {
  void *p = __real_malloc(n);
  if (g_armed) {
    for (int k = 0; k < 2; ++k)
      if (g_count == g_index[k]) g_ptr[k] = p;
    ++g_count;
  }
  return p;
}

void __wrap_free(void *p) {
  for (int k = 0; k < 2; ++k)
    if (p && g_armed && p == g_ptr[k]) {
      memcpy(g_copy[k], p, g_bytes[k]);
      g_ptr[k] = NULL;
    }
  __real_free(p);
}

static void arm(int i0, size_t b0, int i1, size_t b1) {
  if (b0 > sizeof g_copy[0] || b1 > sizeof g_copy[1]) abort();
  g_index[0] = i0;
  g_index[1] = i1;
  g_bytes[0] = b0;
  g_bytes[1] = b1;
  g_ptr[0] = g_ptr[1] = NULL;
  g_count = 0;
  g_armed = 1;
}

/* ---------------------------------------------------------------- the reference's functions */
void convertToarray(const struct svm_node *x, unsigned int *m);
double svm_predict_plain(const struct svm_model *model, unsigned int *m, double *p1, double *p2);
double svm_predict_cpu(const struct svm_model *model, uint32_t c[SIFE_L + 1][SIFE_NMODULI][SIFE_N],
                       const uint32_t msk[SIFE_L][SIFE_NMODULI][SIFE_N], double *p1, double *p2, double *kp,
                       double *dec, double *extract);
double svm_predict_gpu(const struct svm_model *model, uint32_t c[SIFE_L + 1][SIFE_NMODULI][SIFE_N],
                       const uint32_t msk[SIFE_L][SIFE_NMODULI][SIFE_N], double *p1, double *p2, double *kp1,
                       float *kp2, double *dec1, float *dec2, double *extract1);

int cl_n(void) { return SIFE_N; }
int cl_l(void) { return SIFE_L; }

void *cl_load_model(const char *path) { return svm_load_model(path); }

void cl_free_model(void *model) {
  struct svm_model *m = (struct svm_model *)model;
  svm_free_and_destroy_model(&m);
}

int cl_model_info(const void *model, int *nr_class, int *total_sv) {
  const struct svm_model *m = (const struct svm_model *)model;
  *nr_class = m->nr_class;
  *total_sv = m->l;
  return 0;
}

/* the model's arrays: label[nr_class], nsv[nr_class], rho[pairs], coef[nr_class-1][total_sv],
 * sv dense [total_sv][SIFE_L] as convertToarray (main.c:30-41) fills it */
int cl_model_arrays(const void *model, int *label, int *nsv, double *rho, double *coef, uint32_t *sv) {
  const struct svm_model *m = (const struct svm_model *)model;
  const int k = m->nr_class, pairs = k * (k - 1) / 2;
  for (int i = 0; i < k; ++i) {
    label[i] = m->label[i];
    nsv[i] = m->nSV[i];
  }
  for (int p = 0; p < pairs; ++p) rho[p] = m->rho[p];
  for (int j = 0; j + 1 < k; ++j) memcpy(coef + (size_t)j * m->l, m->sv_coef[j], sizeof(double) * m->l);
  for (int i = 0; i < m->l; ++i) convertToarray(m->SV[i], sv + (size_t)i * SIFE_L);
  return 0;
}

double cl_predict_plain(const void *model, unsigned int *msg) {
  double a = 0, b = 0;
  return svm_predict_plain((const struct svm_model *)model, msg, &a, &b);
}

/* svm_predict_cpu ("svm_predict3"): label, dec[pairs] its decision values and kvalue[total_sv]
 * its decoded inner products */
double cl_predict_cpu(const void *model, uint32_t *c, const uint32_t *msk, double *dec, double *kvalue) {
  const struct svm_model *m = (const struct svm_model *)model;
  const int pairs = m->nr_class * (m->nr_class - 1) / 2;
  double t[5] = {0};
  arm(0, sizeof(double) * pairs, 1, sizeof(double) * m->l);
  const double label = svm_predict_cpu(m, (uint32_t(*)[SIFE_NMODULI][SIFE_N])c,
                                       (const uint32_t(*)[SIFE_NMODULI][SIFE_N])msk, t, t + 1, t + 2, t + 3, t + 4);
  g_armed = 0;
  memcpy(dec, g_copy[0], sizeof(double) * pairs);
  memcpy(kvalue, g_copy[1], sizeof(double) * m->l);
  return label;
}

/* svm_predict_gpu ("svm_predict5"): the reference's GPU prediction, which calls
 * rlwe_sife_keygen_gpu and rlwe_sife_decrypt_gmp_gpu -- here those of libcufe_b200.so */
double cl_predict_gpu(const void *model, uint32_t *c, const uint32_t *msk, double *dec, double *kvalue) {
  const struct svm_model *m = (const struct svm_model *)model;
  const int pairs = m->nr_class * (m->nr_class - 1) / 2;
  double t[5] = {0};
  float f[2] = {0};
  arm(0, sizeof(double) * pairs, 4, sizeof(double) * m->l);
  const double label = svm_predict_gpu(m, (uint32_t(*)[SIFE_NMODULI][SIFE_N])c,
                                       (const uint32_t(*)[SIFE_NMODULI][SIFE_N])msk, t, t + 1, t + 2, f, t + 3, f + 1,
                                       t + 4);
  g_armed = 0;
  memcpy(dec, g_copy[0], sizeof(double) * pairs);
  memcpy(kvalue, g_copy[1], sizeof(double) * m->l);
  return label;
}

/* the CPU scheme (src/rlwe_sife.c:32-82, 112-181); seeds from the queue */
void cl_setup(uint32_t *mpk, uint32_t *msk) {
  double t = 0;
  rlwe_sife_setup((uint32_t(*)[SIFE_NMODULI][SIFE_N])mpk, (uint32_t(*)[SIFE_NMODULI][SIFE_N])msk, &t);
}

void cl_encrypt(uint32_t *m, uint32_t *mpk, uint32_t *c) {
  double t = 0;
  rlwe_sife_encrypt(m, (uint32_t(*)[SIFE_NMODULI][SIFE_N])mpk, (uint32_t(*)[SIFE_NMODULI][SIFE_N])c, &t);
}

/* the reference's GPU wrappers (src/rlwe_sife.c:85-109, 184-212), which call
 * rlwe_sife_setup_gpu / rlwe_sife_encrypt_gpu -- here those of libcufe_b200.so */
void cl_setup_gui(uint32_t *mpk, uint32_t *msk) {
  double t1 = 0;
  float t2 = 0;
  rlwe_sife_setup_gui((uint32_t(*)[SIFE_NMODULI][SIFE_N])mpk, (uint32_t(*)[SIFE_NMODULI][SIFE_N])msk, &t1, &t2);
}

void cl_encrypt_gui(uint32_t *m, uint32_t *mpk, uint32_t *c, int repeat) {
  double t1 = 0;
  float t2 = 0;
  rlwe_sife_encrypt_gui(m, (uint32_t(*)[SIFE_NMODULI][SIFE_N])mpk, c, repeat, &t1, &t2);
}
