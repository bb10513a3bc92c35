// scheme.cuh -- device helpers shared by the IPFE kernels (ipfe.cu), the sampler
// (sampler.cu) and the heterogeneous batch kernels (batch.cu).
#pragma once
#include "cufe_internal.cuh"
#include "ntt.cuh"

namespace cufe {

template <int LOGN, int LE = 4>
constexpr int ppc() {  // residue polynomials per CTA (>= 256 threads per CTA)
  return NttPlan<LOGN, LE>::T >= 256 ? 1 : 256 / NttPlan<LOGN, LE>::T;
}

__device__ __forceinline__ void load16(const uint32_t *p, uint32_t (&a)[16]) {
  const uint4 *v = reinterpret_cast<const uint4 *>(p);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint4 t = v[i];
    a[4 * i] = t.x;
    a[4 * i + 1] = t.y;
    a[4 * i + 2] = t.z;
    a[4 * i + 3] = t.w;
  }
}
__device__ __forceinline__ void store16(uint32_t *p, const uint32_t (&a)[16]) {
  uint4 *v = reinterpret_cast<uint4 *>(p);
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = make_uint4(a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]);
}
// E consecutive words (E a multiple of 4, p 16-byte aligned)
template <int E>
__device__ __forceinline__ void load_vec(const uint32_t *p, uint32_t (&a)[E]) {
  const uint4 *v = reinterpret_cast<const uint4 *>(p);
#pragma unroll
  for (int i = 0; i < E / 4; ++i) {
    const uint4 t = v[i];
    a[4 * i] = t.x;
    a[4 * i + 1] = t.y;
    a[4 * i + 2] = t.z;
    a[4 * i + 3] = t.w;
  }
}
template <int E>
__device__ __forceinline__ void store_vec(uint32_t *p, const uint32_t (&a)[E]) {
  uint4 *v = reinterpret_cast<uint4 *>(p);
#pragma unroll
  for (int i = 0; i < E / 4; ++i) v[i] = make_uint4(a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]);
}


struct SchemeArgs {
  RingArgs ra;
  int l;
  uint32_t delta_mod[3], delta_sh[3];
  uint64_t mu[3];
};

__device__ __forceinline__ uint32_t y_residue(uint32_t y, int y_signed, uint32_t q, uint64_t mu) {
  if (!y_signed) return mod_u64(y, mu, q);
  const int32_t ys = (int32_t)y;
  if (ys >= 0) return mod_u64((uint64_t)ys, mu, q);
  const uint32_t r = mod_u64((uint64_t)(-(int64_t)ys), mu, q);
  return r ? q - r : 0u;
}

struct DecodeArgs {
  uint32_t q0, q1, q2;
  uint32_t c1, c1_sh, c2, c2_sh;
  uint64_t mu2;
  uint64_t q01;
  unsigned long long qlo, qhi, hlo, hhi;  // q and floor(q/2) as 128-bit halves
  uint32_t p;
  int n;
};

// crt_reverse_gmp + round_extract_gmp (src/crt.c:46-81, src/rlwe_sife.c:288-332): Garner
// to x in [0, q), then floor(p x / q) + (remainder > floor(q/2)).
__device__ __forceinline__ uint32_t decode_one(uint32_t v0, uint32_t v1, uint32_t v2, const DecodeArgs &d) {
  const uint32_t t1 = mod_red1(v1 + d.q1 - v0 % d.q1, d.q1);
  const uint32_t u1 = shoup_mul(t1, d.c1, d.c1_sh, d.q1);
  const uint64_t x1 = (uint64_t)v0 + (uint64_t)d.q0 * u1;
  const uint32_t xm = mod_u64(x1, d.mu2, d.q2);
  const uint32_t t2 = mod_red1(v2 + d.q2 - xm, d.q2);
  const uint32_t u2 = shoup_mul(t2, d.c2, d.c2_sh, d.q2);
  const u128 Q = ((u128)d.qhi << 64) | d.qlo, H = ((u128)d.hhi << 64) | d.hlo;
  const u128 x = (u128)x1 + (u128)d.q01 * u2;
  const u128 a = x * d.p;
  // quotient < p + 1: estimate in double, correct exactly
  long long qe = (long long)floor((double)x / (double)Q * (double)d.p);
  if (qe < 0) qe = 0;
  u128 prod = (u128)qe * Q;
  while (prod > a) {
    --qe;
    prod -= Q;
  }
  u128 rem = a - prod;
  while (rem >= Q) {
    ++qe;
    rem -= Q;
  }
  if (rem > H) ++qe;
  return (uint32_t)qe;
}


// sum over the CTA of one u64 per thread (values < 2^40); red: blockDim.x/32 words
__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v, uint64_t *red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint64_t t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// index s with off[s] <= g < off[s+1] for a non-decreasing off[0..nseg] with off[0] <= g
template <typename T>
__device__ __forceinline__ uint32_t seg_find(const T *__restrict__ off, uint32_t nseg, uint64_t g) {
  uint32_t lo = 0, hi = nseg;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((uint64_t)__ldg(off + mid) <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

}  // namespace cufe
