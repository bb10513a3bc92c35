// sampler.cuh -- device pieces of the discrete Gaussian samplers (binary sampler: CDT base
// sample, uniform y, Bernoulli rejection), restating src/gauss.c (CPU) and src/sampler.cuh
// (GPU) of the reference bit for bit, including where the reference's behaviour comes from
// its compiled code rather than from the C standard.
#pragma once
#include "cufe_internal.cuh"

namespace cufe {

// Binary-sampler scale factors K_i (sigma_i = K_i * sigma_0, src/gauss.c:11-13)
__host__ __device__ constexpr uint64_t sigma_k(int sig) {
  return sig == 0 ? 266ull : (sig == 1 ? 304214978ull : 608429953ull);
}

// CDT of the base sampler, (low63, high63) of P(x > i) (src/gauss.c:63-73); kept identical
// because every sample bit depends on it.  The high words are also compile-time constants
// (cdt_hi) for the fast path, where two of them are zero and the rest become immediates.
__host__ __device__ constexpr uint64_t cdt_hi(int i) {
  return i == 0 ? 3327841033070651387ull
         : i == 1 ? 380075531178589176ull
         : i == 2 ? 11604843442081400ull
         : i == 3 ? 90134450315532ull
         : i == 4 ? 175786317361ull
         : i == 5 ? 85801740ull
         : i == 6 ? 10472ull
                  : 0ull;
}
static __constant__ uint64_t c_cdt[9][2] = {
    {2200310400551559144ull, cdt_hi(0)}, {7912151619254726620ull, cdt_hi(1)}, {5167367257772081627ull, cdt_hi(2)},
    {5081592746475748971ull, cdt_hi(3)}, {6522074513864805092ull, cdt_hi(4)}, {2579734681240182346ull, cdt_hi(5)},
    {8175784047440310133ull, cdt_hi(6)}, {2947787991558061753ull, cdt_hi(7)}, {22489665999543ull, cdt_hi(8)}};
// 2^f polynomial (src/gauss.c:102-111), kept identical (the Bernoulli compares its bits)
static __constant__ uint64_t c_expc[10] = {0x3e833b70ffa2c5d4ull, 0x3eb4a480fda7e6e1ull, 0x3ef01b254493363full,
                                    0x3f242e0e0aa273ccull, 0x3f55d8a2334ed31bull, 0x3f83b2aa56db0f1aull,
                                    0x3fac6b08e11fc57eull, 0x3fcebfbdff556072ull, 0x3fe62e42fefa7fe6ull,
                                    0x3ff0000000000000ull};


enum : uint32_t {
  kStatusUniformOverrun = 1u,   // a uniform draw ran past the 384-byte refill (reference UB)
  kStatusRefillsExhausted = 2u, // mode A: the precomputed refills did not cover all calls
  kStatusRefillCap = 4u,        // GPU mapping: a thread exceeded kMaxRefillsPerThread refills
  kStatusWideSample = 8u,       // an accepted candidate at or above 2^33 (z = K x + y < 8K keeps it below)
};
// refills one GPU-mapping thread may draw for its 8 samples (needs about 2; 64 has
// probability far below 2^-400 of being exceeded)
constexpr uint32_t kMaxRefillsPerThread = 64;

// CDT base sample (src/gauss.c:122-197, src/sampler.cuh:153-181).  FULL: the 126-bit
// compare of the AVX cdt_sampler (CPU S3); otherwise the high-word compare that
// cdt_sampler64 / cdt_sampler_gpu actually compute.
template <bool FULL>
__device__ __forceinline__ uint32_t cdt_sample(uint64_t r2, uint64_t r1) {
  const uint64_t M = 0x7fffffffffffffffull;
  r2 &= M;
  r1 &= M;
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    uint64_t lt = r2 - c_cdt[i][1];
    if (FULL) lt |= (r1 - c_cdt[i][0]) & (r2 == c_cdt[i][1] ? ~0ull : 0ull);
    x += (uint32_t)(lt >> 63);
  }
  return x;
}
// The high-word compare of cdt_sample<false> from the constant high words, and whether r2
// ties one of them (the FULL compare needs the low words only then), from the same
// differences.
__device__ __forceinline__ uint32_t cdt_sample_hi(uint64_t r2, bool &tie) {
  r2 &= 0x7fffffffffffffffull;
  uint32_t x = 0;
  tie = false;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const uint64_t d = r2 - cdt_hi(i);
    x += (uint32_t)(d >> 63);
    tie |= d == 0;
  }
  return x;
}

// Bernoulli variants (see oracle/cufe_oracle.c bernoulli_lane for the derivation):
// 0 = compiled x86 scalar code (CPU S1/S2), 1 = AVX (CPU S3), 2 = PTX (every GPU kernel).
template <int SIG, int VAR>
__device__ __forceinline__ bool bernoulli_accept(uint64_t xin, uint64_t rm, uint32_t rexp, double kinv) {
  const uint64_t x = xin | 0x4330000000000000ull;
  double vx = (SIG == 0) ? __ull2double_rn(x - 0x4330000000000000ull)
                         : __dsub_rn(__longlong_as_double((long long)x), 4503599627370496.0);
  vx = __dmul_rn(vx, kinv);
  const double fl = floor(vx);
  const double t = __dadd_rn(fl, 6755399441055744.0);
  uint64_t vtu;
  if (VAR == 1) {
    vtu = ((uint64_t)__double_as_longlong(t) - 0x4338000000000000ull) << 52;
  } else {
    long long ti;
    if (t >= 9223372036854775808.0)
      ti = (VAR == 2) ? 0x7fffffffffffffffll : (long long)0x8000000000000000ull;
    else if (t < -9223372036854775808.0)
      ti = (long long)0x8000000000000000ull;
    else
      ti = __double2ll_rz(t);
    vtu = ((uint64_t)ti - 0x0018000000000000ull) << 52;
  }
  const double f = __dsub_rn(vx, fl);
  double s = __fma_rn(__longlong_as_double((long long)c_expc[0]), f, __longlong_as_double((long long)c_expc[1]));
#pragma unroll
  for (int c = 2; c < 10; ++c) s = __fma_rn(s, f, __longlong_as_double((long long)c_expc[c]));
  const int64_t vres = (int64_t)(vtu + (uint64_t)__double_as_longlong(s));
  const int64_t rmant = (vres & ((1ll << 52) - 1)) | (1ll << 52);
  const int64_t rexpo =
      (VAR == 1 ? (int64_t)((uint64_t)vres >> 52) : (vres >> 52)) + (19 - 1023 + 1);
  int64_t rp;
  if (VAR != 0)
    rp = (rexpo >= 0 && rexpo < 64) ? (int64_t)(1ull << rexpo) : 0;
  else if (SIG == 0 || rexpo >= 0)
    rp = (int64_t)(1ull << (rexpo & 63));
  else
    rp = 0;
  const int64_t r_exp = (int64_t)(((rm >> 53) & 0x7ffull) | ((uint64_t)rexp << 11));
  const int64_t r_mant = (int64_t)(rm & ((1ull << 53) - 1));
  const bool eq1 = vres == (1023ll << 52);
  return eq1 || ((((uint64_t)(r_mant - rmant) & (uint64_t)(r_exp - rp)) >> 63) != 0);
}

// uniform y in [0, K): 32-bit rejection then Barrett (src/gauss.c:578-703)
template <int SIG>
__device__ __forceinline__ bool uniform_ok(uint32_t x) {
  constexpr uint64_t K = sigma_k(SIG), BF = (1ull << 32) / K, UQ = K * BF;
  return (uint64_t)x < UQ;
}
template <int SIG>
__device__ __forceinline__ uint32_t uniform_reduce(uint32_t x32) {
  constexpr uint64_t K = sigma_k(SIG), BF = (1ull << 32) / K;
  uint64_t x = x32;
  x = x - ((((x * BF) >> 32) + 1) * K);
  x = x + (x >> 63) * K;
  return (uint32_t)x;
}

// one candidate: z = K x + y, Bernoulli input (uint32)(z + K x) * y (src/gauss.c:836-850)
template <int SIG, int VAR>
__device__ __forceinline__ bool candidate(uint32_t x, uint32_t y, uint64_t rm, uint32_t rexp, double kinv,
                                          uint64_t &z) {
  constexpr uint64_t K = sigma_k(SIG);
  const uint64_t kx = (uint64_t)x * K;
  z = kx + y;
  const uint64_t vb = (uint64_t)(uint32_t)(z + kx) * (uint64_t)y;
  return bernoulli_accept<SIG, VAR>(vb, rm, rexp, kinv);
}

// accept iff Bernoulli bit and (z != 0 or negative sign) (src/gauss.c:887)
__device__ __forceinline__ bool accept_final(bool b, uint64_t z, uint32_t k) { return b && (z != 0 || k != 0); }

}  // namespace cufe
