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

typedef unsigned __int128 u128;

constexpr int kMaxModuli = 6;
constexpr int kMaxLogN = 13;

// Device-visible description of an RNS ring Z_q[X]/(X^n+1): the primes and the
// bit-reversed twiddle tables (psi[m+i] = psi^{bitrev(m+i)}, the layout of the
// reference's consts.h), each entry interleaved with its Shoup companion
// floor(w * 2^32 / q) so that one 8- or 16-byte load fetches one or two twiddles.
struct RingArgs {
  int n, logn, k;
  uint32_t q[kMaxModuli];
  uint32_t ninv[kMaxModuli], ninv_sh[kMaxModuli];  // n^-1
  uint32_t w1n[kMaxModuli], w1n_sh[kMaxModuli];    // psi_inv[1] * n^-1 (last inverse stage)
  uint32_t qr[kMaxModuli];                          // floor(2^32 / q)
  const uint2 *psi2, *ipsi2;                       // [k][n] (w, w_shoup) each
  int pp_fwd, pp_inv;  // NTT kernel variant per direction (1..CUFE_NTT_VARIANTS), set by the tuner
};

// ------------------------------------------------------------------ arithmetic
// All residues are kept canonical in [0, q) with q < 2^31.

// The reductions are min(x, x - q) over uint32 (x - q wraps above x when x < q), written
// with the fused add-and-min __viaddmin_u32(a, b, c) = min(a + b, c).
__device__ __forceinline__ uint32_t mod_red1(uint32_t x, uint32_t q) {  // x < 2q
  return __viaddmin_u32(x, 0u - q, x);
}
__device__ __forceinline__ uint32_t mod_add(uint32_t a, uint32_t b, uint32_t q) {  // a, b < q
  return __viaddmin_u32(a, b, a + b - q);
}
__device__ __forceinline__ uint32_t mod_sub(uint32_t a, uint32_t b, uint32_t q) {  // a, b < q
  const uint32_t d = a - b;
  return __viaddmin_u32(d, q, d);
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
