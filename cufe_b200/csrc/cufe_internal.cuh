// cufe_internal.cuh -- shared device/host definitions of the cufe_b200 library.
//
// Residue polynomials are laid out as in the reference (src/rlwe_sife.h:10-26):
// [poly][modulus][n] uint32, so residue polynomial r (flat index) has modulus r % k.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/cufe_b200.h"

namespace cufe {

constexpr int kMaxModuli = 6;
constexpr int kMaxLogN = 13;

// Device-visible description of an RNS ring Z_q[X]/(X^n+1): the primes and the
// bit-reversed twiddle tables (psi[m+i] = psi^{bitrev(m+i)}, the layout of the
// reference's consts.h) with their Shoup companions floor(w * 2^32 / q).
struct RingArgs {
  int n, logn, k;
  uint32_t q[kMaxModuli];
  uint32_t ninv[kMaxModuli], ninv_sh[kMaxModuli];  // n^-1
  uint32_t w1n[kMaxModuli], w1n_sh[kMaxModuli];    // psi_inv[1] * n^-1 (last inverse stage)
  const uint32_t *psi, *psi_sh, *ipsi, *ipsi_sh;   // [k][n] each
};

// ------------------------------------------------------------------ arithmetic
// All residues are kept canonical in [0, q) with q < 2^31.

__device__ __forceinline__ uint32_t mod_red1(uint32_t x, uint32_t q) {  // x < 2q
  return min(x, x - q);
}
__device__ __forceinline__ uint32_t mod_add(uint32_t a, uint32_t b, uint32_t q) {
  return mod_red1(a + b, q);
}
__device__ __forceinline__ uint32_t mod_sub(uint32_t a, uint32_t b, uint32_t q) {
  return mod_red1(a - b + q, q);
}
// Shoup: a * w mod q for a constant w with wsh = floor(w * 2^32 / q); any a < 2^32.
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t a, uint32_t w, uint32_t wsh, uint32_t q) {
  uint32_t hi = __umulhi(a, wsh);
  return a * w - hi * q;  // in [0, 2q)
}
__device__ __forceinline__ uint32_t shoup_mul(uint32_t a, uint32_t w, uint32_t wsh, uint32_t q) {
  return mod_red1(shoup_lazy(a, w, wsh, q), q);
}
// x mod q for a 64-bit x, with mu = floor(2^64 / q) (q < 2^31, q not a power of two)
__device__ __forceinline__ uint32_t mod_u64(uint64_t x, uint64_t mu, uint32_t q) {
  uint64_t qe = __umul64hi(x, mu);
  uint64_t r = x - qe * q;  // < 2q
  return (uint32_t)(r >= q ? r - q : r);
}

// ------------------------------------------------------------------ host helpers

inline uint32_t shoup_of(uint32_t w, uint32_t q) {
  return (uint32_t)(((uint64_t)w << 32) / q);
}

struct CudaError {
  cudaError_t e;
  const char *where;
};

#define CUFE_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess) {                                                             \
      ::cufe::set_last_error(std::string(#call) + ": " + cudaGetErrorString(_e));       \
      return CUFE_ERR_CUDA;                                                              \
    }                                                                                    \
  } while (0)

void set_last_error(const std::string &msg);

}  // namespace cufe
