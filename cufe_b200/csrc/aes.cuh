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

// rounds R0..14 on the state after round R0 - 1 (R0 = 1: after the initial AddRoundKey)
template <int R0>
__device__ __forceinline__ void aes256_rounds_from(uint32_t &s0, uint32_t &s1, uint32_t &s2, uint32_t &s3,
                                                   const uint32_t (&rk)[60], const AesCtx &c) {
#pragma unroll
  for (int r = R0; r < 14; ++r) {
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

// rounds 1..14 on a state that already holds input ^ rk[0..3]
__device__ __forceinline__ void aes256_rounds(uint32_t &s0, uint32_t &s1, uint32_t &s2, uint32_t &s3,
                                              const uint32_t (&rk)[60], const AesCtx &c) {
  aes256_rounds_from<1>(s0, s1, s2, s3, rk, c);
}

// Counter caching for the CPU mapping with nonce 0: the input block is 0^12 || BE32(ctr), so
// after the initial AddRoundKey only state word 3 depends on ctr.  In round 1 each output
// word takes exactly one byte of word 3 (T3 of its low byte for word 0, T2/T1/T0 of the
// higher bytes for words 1..3); for counters with equal upper 24 bits, words 1..3 after round
// 1 are therefore fixed and only word 0 varies, and in round 2 each output word takes one byte
// of word 0 and three fixed bytes.  k0..k3: the ctr-independent part of round 1 (per key);
// c0..c3: the fixed part of round 2 for the upper counter bits `hi` (recomputed when they
// change).  Per block, rounds 1 and 2 then take 1 + 4 table lookups instead of 32.
// The round-2 keys rk[8..11] are needed only when `hi` changes (about every 10 refills), so
// they are read from the key schedule in global memory (rkg) and occupy no registers between
// blocks.
struct CtrCache {
  uint32_t k0, k1, k2, k3, c0, c1, c2, c3, hi;
};

__device__ __forceinline__ void ctr_cache_key(CtrCache &cc, const uint32_t (&rk)[60], const AesCtx &c) {
  const uint32_t s0 = rk[0], s1 = rk[1], s2 = rk[2];
  cc.k0 = te<0>(c, taddr<3>(c, s0)) ^ te<1>(c, taddr<2>(c, s1)) ^ te<2>(c, taddr<1>(c, s2)) ^ rk[4];
  cc.k1 = te<0>(c, taddr<3>(c, s1)) ^ te<1>(c, taddr<2>(c, s2)) ^ te<3>(c, taddr<0>(c, s0)) ^ rk[5];
  cc.k2 = te<0>(c, taddr<3>(c, s2)) ^ te<2>(c, taddr<1>(c, s0)) ^ te<3>(c, taddr<0>(c, s1)) ^ rk[6];
  cc.k3 =
      te<1>(c, taddr<2>(c, s0)) ^ te<2>(c, taddr<1>(c, s1)) ^ te<3>(c, taddr<0>(c, s2)) ^ rk[7];
  cc.hi = 0xffffffffu;  // no counter cached
}

// the keystream block of counter ctr (nonce 0), output as in aes256_ctr_block; rkg: the same
// key schedule as rk, in global memory
__device__ __forceinline__ void aes256_ctr_block_cached(uint32_t (&o)[4], uint32_t ctr, const uint32_t (&rk)[60],
                                                        const uint32_t *__restrict__ rkg, const AesCtx &c,
                                                        CtrCache &cc) {
  const uint32_t w3 = ctr ^ rk[3];
  if ((ctr >> 8) != cc.hi) {
    cc.hi = ctr >> 8;
    const uint32_t u1 = cc.k1 ^ te<2>(c, taddr<1>(c, w3));
    const uint32_t u2 = cc.k2 ^ te<1>(c, taddr<2>(c, w3));
    const uint32_t u3 = cc.k3 ^ te<0>(c, taddr<3>(c, w3));
    const uint4 k2 = __ldg(reinterpret_cast<const uint4 *>(rkg + 8));
    cc.c0 = te<1>(c, taddr<2>(c, u1)) ^ te<2>(c, taddr<1>(c, u2)) ^ te<3>(c, taddr<0>(c, u3)) ^ k2.x;
    cc.c1 = te<0>(c, taddr<3>(c, u1)) ^ te<1>(c, taddr<2>(c, u2)) ^ te<2>(c, taddr<1>(c, u3)) ^ k2.y;
    cc.c2 = te<0>(c, taddr<3>(c, u2)) ^ te<1>(c, taddr<2>(c, u3)) ^ te<3>(c, taddr<0>(c, u1)) ^ k2.z;
    cc.c3 = te<0>(c, taddr<3>(c, u3)) ^ te<2>(c, taddr<1>(c, u1)) ^ te<3>(c, taddr<0>(c, u2)) ^ k2.w;
  }
  const uint32_t a0 = cc.k0 ^ te<3>(c, taddr<0>(c, w3));
  uint32_t s0 = cc.c0 ^ te<0>(c, taddr<3>(c, a0)), s1 = cc.c1 ^ te<3>(c, taddr<0>(c, a0));
  uint32_t s2 = cc.c2 ^ te<2>(c, taddr<1>(c, a0)), s3 = cc.c3 ^ te<1>(c, taddr<2>(c, a0));
  aes256_rounds_from<3>(s0, s1, s2, s3, rk, c);
  o[0] = s0;
  o[1] = s1;
  o[2] = s2;
  o[3] = s3;
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
