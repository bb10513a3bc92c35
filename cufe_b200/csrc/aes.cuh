// aes.cuh -- AES-256 block function for the samplers' keystreams (FIPS-197).
//
// T-table formulation (one SubBytes+ShiftRows+MixColumns round = 16 table lookups + XORs).
// Each of the four 256-entry tables is replicated once per shared-memory bank so a warp's 32
// lookups never conflict: entry x of table t for lane L lives at byte
//   (t >> 1) * 64 KiB + x * 256 + (t & 1) * 128 + L * 4,
// so the lookup address is one PRMT of the state word with the per-lane constant L*4 (the
// table offset is an immediate of the LDS).  128 KiB of shared memory per CTA.
// Round keys are 60 big-endian words in registers; an all-zero key schedule is valid (the
// reference CPU path's uninitialised AES contexts).
#pragma once
#include "cufe_internal.cuh"

namespace cufe {

constexpr int kAesSmemBytes = 131072;

// S-box, uploaded by sampler_init_device (computed from GF(2^8) inversion + affine map)
static __constant__ uint8_t c_sbox[256];

__device__ __forceinline__ uint32_t xtime_u8(uint32_t b) {
  return ((b << 1) ^ ((b & 0x80u) ? 0x1bu : 0u)) & 0xffu;
}

// fill the replicated tables (all threads of the CTA; caller syncs)
__device__ __forceinline__ void aes_fill_tables(uint8_t *smem) {
  uint32_t *w = reinterpret_cast<uint32_t *>(smem);
  for (int i = threadIdx.x + threadIdx.y * blockDim.x; i < kAesSmemBytes / 4;
       i += blockDim.x * blockDim.y) {
    const int region = i >> 14, x = (i >> 6) & 255, t1 = (i >> 5) & 1;
    const int t = region * 2 + t1;
    const uint32_t s = c_sbox[x];
    const uint32_t te0 = (xtime_u8(s) << 24) | (s << 16) | (s << 8) | (xtime_u8(s) ^ s);
    w[i] = t == 0 ? te0 : __funnelshift_r(te0, te0, 8 * t);
  }
}

struct AesCtx {
  const uint8_t *base;  // shared-memory tables
  uint32_t laneoff;     // (lane & 31) * 4
};

template <int T>
__device__ __forceinline__ uint32_t te(const AesCtx &c, uint32_t addr) {
  return *reinterpret_cast<const uint32_t *>(c.base + addr + (T >> 1) * 65536 + (T & 1) * 128);
}
// byte b (3 = most significant) of s as a table address
template <int B>
__device__ __forceinline__ uint32_t taddr(const AesCtx &c, uint32_t s) {
  return __byte_perm(s, c.laneoff, 0x5504 | (B << 4));
}

// rounds 1..14 on a state that already holds input ^ rk[0..3]
__device__ __forceinline__ void aes256_rounds(uint32_t &s0, uint32_t &s1, uint32_t &s2, uint32_t &s3,
                                              const uint32_t (&rk)[60], const AesCtx &c) {
#pragma unroll
  for (int r = 1; r < 14; ++r) {
    const uint32_t t0 = te<0>(c, taddr<3>(c, s0)) ^ te<1>(c, taddr<2>(c, s1)) ^
                        te<2>(c, taddr<1>(c, s2)) ^ te<3>(c, taddr<0>(c, s3)) ^ rk[4 * r];
    const uint32_t t1 = te<0>(c, taddr<3>(c, s1)) ^ te<1>(c, taddr<2>(c, s2)) ^
                        te<2>(c, taddr<1>(c, s3)) ^ te<3>(c, taddr<0>(c, s0)) ^ rk[4 * r + 1];
    const uint32_t t2 = te<0>(c, taddr<3>(c, s2)) ^ te<1>(c, taddr<2>(c, s3)) ^
                        te<2>(c, taddr<1>(c, s0)) ^ te<3>(c, taddr<0>(c, s1)) ^ rk[4 * r + 2];
    const uint32_t t3 = te<0>(c, taddr<3>(c, s3)) ^ te<1>(c, taddr<2>(c, s0)) ^
                        te<2>(c, taddr<1>(c, s1)) ^ te<3>(c, taddr<0>(c, s2)) ^ rk[4 * r + 3];
    s0 = t0;
    s1 = t1;
    s2 = t2;
    s3 = t3;
  }
  // final round: S-box bytes taken from the tables (Te2 byte 3, Te3 byte 2, Te0 byte 1, Te1 byte 0)
  const uint32_t o0 = (te<2>(c, taddr<3>(c, s0)) & 0xff000000u) ^ (te<3>(c, taddr<2>(c, s1)) & 0x00ff0000u) ^
                      (te<0>(c, taddr<1>(c, s2)) & 0x0000ff00u) ^ (te<1>(c, taddr<0>(c, s3)) & 0x000000ffu) ^ rk[56];
  const uint32_t o1 = (te<2>(c, taddr<3>(c, s1)) & 0xff000000u) ^ (te<3>(c, taddr<2>(c, s2)) & 0x00ff0000u) ^
                      (te<0>(c, taddr<1>(c, s3)) & 0x0000ff00u) ^ (te<1>(c, taddr<0>(c, s0)) & 0x000000ffu) ^ rk[57];
  const uint32_t o2 = (te<2>(c, taddr<3>(c, s2)) & 0xff000000u) ^ (te<3>(c, taddr<2>(c, s3)) & 0x00ff0000u) ^
                      (te<0>(c, taddr<1>(c, s0)) & 0x0000ff00u) ^ (te<1>(c, taddr<0>(c, s1)) & 0x000000ffu) ^ rk[58];
  const uint32_t o3 = (te<2>(c, taddr<3>(c, s3)) & 0xff000000u) ^ (te<3>(c, taddr<2>(c, s0)) & 0x00ff0000u) ^
                      (te<0>(c, taddr<1>(c, s1)) & 0x0000ff00u) ^ (te<1>(c, taddr<0>(c, s2)) & 0x000000ffu) ^ rk[59];
  s0 = o0;
  s1 = o1;
  s2 = o2;
  s3 = o3;
}

// One keystream block of the CPU counter mapping (src/aes256ctr.c:13-81): input
// BE16(nonce) || 0^10 || BE32(ctr); output as four big-endian words.
__device__ __forceinline__ void aes256_ctr_block(uint32_t (&o)[4], uint32_t nonce_word, uint32_t ctr,
                                                 const uint32_t (&rk)[60], const AesCtx &c) {
  uint32_t s0 = nonce_word ^ rk[0], s1 = rk[1], s2 = rk[2], s3 = ctr ^ rk[3];
  aes256_rounds(s0, s1, s2, s3, rk, c);
  o[0] = s0;
  o[1] = s1;
  o[2] = s2;
  o[3] = s3;
}

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

}  // namespace cufe
