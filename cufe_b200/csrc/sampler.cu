// sampler.cu -- AES-256-CTR keystreams and the discrete Gaussian / uniform samplers.
//
// Two counter-to-sample mappings are implemented, both bit-exact:
//
//  * CPU mapping (src/gauss.c + src/aes256ctr.c): one AES-CTR stream per context; every
//    gaussian_sampler_* call consumes 384-byte refills (24 counter blocks) in order, takes
//    the accepted candidates in order and drops the rest of its last refill.  The stream is
//    sequential by construction, so it is computed in three parallel phases: (1) every
//    refill's 8 candidates and accept mask for a generous refill range (the AES work, one
//    thread per refill), (2) a per-stream exclusive scan of accept counts and a one-warp
//    walk that finds where each call starts (each call starts at a fresh refill), (3) a
//    scatter of the accepted candidates to their coefficient positions as residues.
//  * GPU mapping (src/sample_gpu.cu, src/AES.cuh): thread t of polynomial p owns coefficients
//    8t..8t+7 and draws chained-AES refills from counter p*5*T*24 + rep*T*24 + t*24.
#include "aes.cuh"
#include "sampler.cuh"
#include "sampler_host.h"
#include "scheme.cuh"
#include "prof.h"

#include <algorithm>
#include <cmath>

namespace cufe {

namespace {

__device__ __forceinline__ uint64_t le64_of(uint32_t be_lo, uint32_t be_hi) {
  return (uint64_t)bswap32(be_lo) | ((uint64_t)bswap32(be_hi) << 32);
}

// ------------------------------------------------------------------ CPU mapping, phase 1

// one keystream block of the CPU mapping from round keys in global memory (rare paths)
__device__ __noinline__ void ctr_block_g(uint32_t (&W)[4], uint32_t ctr, const uint32_t *__restrict__ rkg,
                                         const AesCtx &c) {
  uint32_t rk[60];
#pragma unroll
  for (int i = 0; i < 60; ++i) rk[i] = __ldg(rkg + i);
  aes256_ctr_block(W, 0u, ctr, rk, c);
}

// uniform draws when the first 10 words hold fewer than 8 accepted ones (at least 3 of 10
// draws rejected: about 7e-5 per refill for sigma_2 and sigma_3, whose rejection rate is
// 1 - 7 K / 2^32 = 0.84%; far less for sigma_1): rescan bytes 200.. with the rejection loop of
// src/gauss.c:578-703, regenerating blocks as needed
template <int SIG>
__device__ __noinline__ void uniform_slow(uint32_t *y, int ystride, uint32_t cb, const uint32_t *__restrict__ rkg,
                                          const AesCtx &c, uint32_t *status) {
  int w = 0, have_blk = -1;
  uint32_t W[4] = {0, 0, 0, 0};
  for (int j = 0; j < 8; ++j) {
    uint32_t x = 0;
    for (;;) {
      if (w >= 46) {  // would read beyond the 384-byte refill: undefined in the reference
        atomicOr(status, kStatusUniformOverrun);
        x = 0;
        break;
      }
      const int byte = 200 + 4 * w, blk = byte >> 4;
      if (blk != have_blk) {
        ctr_block_g(W, cb + (uint32_t)blk, rkg, c);
        have_blk = blk;
      }
      const int wi = (byte >> 2) & 3;
      x = bswap32(wi == 0 ? W[0] : wi == 1 ? W[1] : wi == 2 ? W[2] : W[3]);
      ++w;
      if (uniform_ok<SIG>(x)) break;
    }
    y[j * ystride] = uniform_reduce<SIG>(x);
  }
}

// 126-bit CDT compare of the CPU S3 for one lane whose high word ties a table entry: the
// low word (bytes 8 lane.. of r, or of r + 100 for lanes 4..7) is regenerated here
__device__ __noinline__ uint32_t cdt_full_slow(int lane, uint64_t r2, uint32_t cb, const uint32_t *__restrict__ rkg,
                                               const AesCtx &c) {
  const int off = (lane < 4 ? 0 : 100) + 8 * (lane & 3);
  uint32_t W[4], lo, hi;
  ctr_block_g(W, cb + (uint32_t)(off >> 4), rkg, c);
  const int w0 = (off >> 2) & 3;
  lo = w0 == 0 ? W[0] : w0 == 1 ? W[1] : w0 == 2 ? W[2] : W[3];
  const int off2 = off + 4;
  if ((off2 >> 4) != (off >> 4)) ctr_block_g(W, cb + (uint32_t)(off2 >> 4), rkg, c);
  const int w1 = (off2 >> 2) & 3;
  hi = w1 == 0 ? W[0] : w1 == 1 ? W[1] : w1 == 2 ? W[2] : W[3];
  return cdt_sample<true>(r2, (uint64_t)bswap32(lo) | ((uint64_t)bswap32(hi) << 32));
}

template <bool FULL>
__device__ __forceinline__ uint32_t cdt_lane(int lane, uint64_t r2, uint32_t cb, const uint32_t *rkg,
                                             const AesCtx &c) {
  bool tie;
  const uint32_t x = cdt_sample_hi(r2, tie);
  if (FULL && tie) return cdt_full_slow(lane, r2, cb, rkg, c);
  return x;
}

// Blocks of one refill that the fast path reads (16-byte block b = bytes 16b..16b+15, word w
// = bytes 4w..4w+3): 2, 3 (CDT high words of lanes 0..3, words 8..15), 4, 5, 6 (Bernoulli
// words 16..24), 8..12 (CDT high words and Bernoulli words of lanes 4..7, words 33..49),
// 12..14 (the first 10 uniform words from byte 200, words 50..59) and 17 (sign byte 280,
// word 70): 13 of the refill's 24 blocks.  Blocks 0, 1, 7 hold only the low CDT words, which
// S1/S2 never use and S3 uses only on ties; blocks 15 and 16 hold uniform words 60..67, needed
// only when fewer than 8 of the first 10 words are accepted.  Both rare cases regenerate what
// they need on their slow paths.
//
// The blocks are computed in the order below and each is consumed as soon as it exists, so a
// refill never buffers its keystream: the uniform words and the sign byte first (every
// candidate needs its y and sign bit), then the exponent word of lanes 0..3, and from there
// every CDT sample and every candidate the moment its last word arrives.  All live values
// (the 8 y, the packed CDT samples, a few words carried to the next block, the outputs) are
// registers; a buffered keystream had to live in local memory, whose traffic took 6% of the
// L1 data pipe that the table lookups saturate and missed L1 on a third of its loads.
constexpr int kRefillBlocks = 13;
__constant__ uint8_t c_refill_order[kRefillBlocks] = {12, 13, 14, 17, 6, 2, 3, 4, 5, 8, 9, 10, 11};

constexpr int kCandThreads = 512;  // 1 CTA (128 KiB of tables) per SM; 128 registers per thread

// Word W (0..9) of the branch-free uniform scan (src/gauss.c:578-703): the first 8 accepted
// words from byte 200 become y[0..7], kept in registers (the same 8 words in a shared-memory
// slot measured 17% slower on the whole kernel).  With at most 2 of the 10 words rejected
// (otherwise the slow path redoes the scan) word W lands in slot W - rej, rej = rejections
// before it, so only the slots W-2..W are candidates (3 selects per word, not 8); slots past
// 7 are dropped, as the reference's loop stops at 8 accepted words.
template <int SIG, int W>
__device__ __forceinline__ void uniform_step(uint32_t (&y)[8], uint32_t &rej, uint32_t be_word) {
  const uint32_t v = bswap32(be_word);
  const bool ok = uniform_ok<SIG>(v);
  const uint32_t r = uniform_reduce<SIG>(v);
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (W - k >= 0 && W - k < 8) y[W - k] = (ok && rej == (uint32_t)k) ? r : y[W - k];
  rej += ok ? 0u : 1u;
}

// Candidate ln of the refill (src/gauss.c:836-890): CDT sample x (packed 4 bits per lane in
// xp), uniform y, Bernoulli words rm (bytes 64 + 8 li + 100 h) and exponent byte, sign bit ln
// of k8.  |value| = z < 8K < 2^33 is kept as its low word (returned) and, in `bits`, its accept
// bit (bit ln), its bit 32 (bit 8 + ln) and bit 16 if an accepted z ever reaches 2^33.
template <int SIG, int VAR>
__device__ __forceinline__ uint32_t refill_candidate(int ln, uint32_t xp, uint32_t y, uint32_t rm_lo,
                                                     uint32_t rm_hi, uint32_t ewrd, uint32_t k8, double kinv,
                                                     uint32_t &bits) {
  const uint32_t x = (xp >> (4 * ln)) & 15u;
  const uint32_t rexp = (ewrd >> (24 - 8 * (ln & 3))) & 0xffu;
  uint64_t z;
  const bool b = candidate<SIG, VAR>(x, y, le64_of(rm_lo, rm_hi), rexp, kinv, z);
  const uint32_t a = accept_final(b, z, (k8 >> ln) & 1u);
  bits |= (a << ln) | ((uint32_t)((z >> 32) & 1u) << (8 + ln)) | ((a & (uint32_t)((z >> 33) != 0)) << 16);
  return (uint32_t)z;
}

template <int SIG, bool FULL, int VAR>
__global__ void __launch_bounds__(kCandThreads, 1)
    k_cand_cpu(const uint32_t *__restrict__ rkeys, SegDev sg, double kinv, uint32_t *__restrict__ cand_lo,
               uint8_t *__restrict__ amask, uint16_t *__restrict__ chs, uint32_t *__restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  aes_fill_tables(smem);
  __syncthreads();
  const AesCtx c{smem, (threadIdx.x & 31u) * 4u};
  // the host keeps the flattened refill count below 2^32 - 2^24 (no wrap of g)
  const uint32_t total = (uint32_t)__ldg(sg.roff + sg.nstreams);
  uint32_t rk[60];
  uint32_t st = 0;
  uint32_t lo = 1, hi = 0;  // refill range of stream st (empty: forces the first lookup)
  CtrCache cc;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    if (g < lo || g >= hi) {
      st = seg_find(sg.roff, sg.nstreams, g);
      lo = (uint32_t)__ldg(sg.roff + st);
      hi = (uint32_t)__ldg(sg.roff + st + 1);
#pragma unroll
      for (int i = 0; i < 60; ++i) rk[i] = __ldg(rkeys + (size_t)st * 60 + i);
      ctr_cache_key(cc, rk, c);
    }
    const uint32_t *rkg = rkeys + (size_t)st * 60;  // the key schedule again, for rare paths
    const uint32_t t = g - lo;
    const uint32_t cb = t * 24u;
    uint32_t y[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) y[j] = 0;
    uint32_t rej = 0, k8 = 0, xp = 0, w24 = 0, w48 = 0, w49 = 0, carry = 0, lo0 = 0, lo1 = 0;
    uint32_t bits = 0;  // accept mask, bits 32 (<< 8), wide flag (bit 16)
    // one AES body for all 13 blocks (keeps the loop inside the instruction cache); the
    // consumer of each block is selected by the (warp-uniform) step
#pragma unroll 1
    for (int step = 0; step < kRefillBlocks; ++step) {
      uint32_t W[4];
      aes256_ctr_block_cached(W, cb + c_refill_order[step], rk, rkg, c, cc);
      switch (step) {
        case 0:  // block 12: words 48 (rm high word of lane 7), 49 (exponents of lanes 4..7), 50, 51
          w48 = W[0];
          w49 = W[1];
          uniform_step<SIG, 0>(y, rej, W[2]);
          uniform_step<SIG, 1>(y, rej, W[3]);
          break;
        case 1:  // block 13: uniform words 52..55
          uniform_step<SIG, 2>(y, rej, W[0]);
          uniform_step<SIG, 3>(y, rej, W[1]);
          uniform_step<SIG, 4>(y, rej, W[2]);
          uniform_step<SIG, 5>(y, rej, W[3]);
          break;
        case 2:  // block 14: uniform words 56..59; fewer than 8 of the 10 accepted: slow path
          uniform_step<SIG, 6>(y, rej, W[0]);
          uniform_step<SIG, 7>(y, rej, W[1]);
          uniform_step<SIG, 8>(y, rej, W[2]);
          uniform_step<SIG, 9>(y, rej, W[3]);
          if (rej > 2) {
            uint32_t ys[8];
            uniform_slow<SIG>(ys, 1, cb, rkg, c, status);
#pragma unroll
            for (int j = 0; j < 8; ++j) y[j] = ys[j];
          }
          break;
        case 3:  // block 17: word 70 holds the sign byte 280
          k8 = bswap32(W[2]) & 0xffu;
          break;
        case 4:  // block 6: word 24, the exponent bytes of lanes 0..3
          w24 = W[0];
          break;
        case 5:  // block 2: CDT high words of lanes 0 (words 8, 9) and 1 (10, 11)
          xp |= cdt_lane<FULL>(0, le64_of(W[0], W[1]), cb, rkg, c);
          xp |= cdt_lane<FULL>(1, le64_of(W[2], W[3]), cb, rkg, c) << 4;
          break;
        case 6:  // block 3: lanes 2 (12, 13) and 3 (14, 15)
          xp |= cdt_lane<FULL>(2, le64_of(W[0], W[1]), cb, rkg, c) << 8;
          xp |= cdt_lane<FULL>(3, le64_of(W[2], W[3]), cb, rkg, c) << 12;
          break;
        case 7:  // block 4: Bernoulli words of lanes 0 (16, 17) and 1 (18, 19)
          lo0 = refill_candidate<SIG, VAR>(0, xp, y[0], W[0], W[1], w24, k8, kinv, bits);
          lo1 = refill_candidate<SIG, VAR>(1, xp, y[1], W[2], W[3], w24, k8, kinv, bits);
          break;
        case 8: {  // block 5: lanes 2 (20, 21) and 3 (22, 23); candidates 0..3 complete
          const uint32_t lo2 = refill_candidate<SIG, VAR>(2, xp, y[2], W[0], W[1], w24, k8, kinv, bits);
          const uint32_t lo3 = refill_candidate<SIG, VAR>(3, xp, y[3], W[2], W[3], w24, k8, kinv, bits);
          reinterpret_cast<uint4 *>(cand_lo + (size_t)g * 8)[0] = make_uint4(lo0, lo1, lo2, lo3);
          break;
        }
        case 9:  // block 8: CDT words of lane 4 (33, 34); word 35 starts lane 5
          xp |= cdt_lane<FULL>(4, le64_of(W[1], W[2]), cb, rkg, c) << 16;
          carry = W[3];
          break;
        case 10:  // block 9: lanes 5 (35, 36) and 6 (37, 38); word 39 starts lane 7
          xp |= cdt_lane<FULL>(5, le64_of(carry, W[0]), cb, rkg, c) << 20;
          xp |= cdt_lane<FULL>(6, le64_of(W[1], W[2]), cb, rkg, c) << 24;
          carry = W[3];
          break;
        case 11:  // block 10: lane 7 CDT (39, 40); Bernoulli words of lane 4 (41, 42); 43 starts lane 5
          xp |= cdt_lane<FULL>(7, le64_of(carry, W[0]), cb, rkg, c) << 28;
          lo0 = refill_candidate<SIG, VAR>(4, xp, y[4], W[1], W[2], w49, k8, kinv, bits);
          carry = W[3];
          break;
        default: {  // block 11: Bernoulli words of lanes 5 (43, 44), 6 (45, 46), 7 (47, 48)
          const uint32_t lo5 = refill_candidate<SIG, VAR>(5, xp, y[5], carry, W[0], w49, k8, kinv, bits);
          const uint32_t lo6 = refill_candidate<SIG, VAR>(6, xp, y[6], W[1], W[2], w49, k8, kinv, bits);
          const uint32_t lo7 = refill_candidate<SIG, VAR>(7, xp, y[7], W[3], w48, w49, k8, kinv, bits);
          reinterpret_cast<uint4 *>(cand_lo + (size_t)g * 8)[1] = make_uint4(lo0, lo5, lo6, lo7);
          break;
        }
      }
    }
    amask[g] = (uint8_t)bits;
    chs[g] = (uint16_t)(((bits >> 8) & 0xffu) | (k8 << 8));
    if (bits & 0x10000u) atomicOr(status, kStatusWideSample);
  }
}

// ------------------------------------------------------------------ CPU mapping, phase 2

constexpr int kScanTile = 4096;  // refills per scan tile (512 threads x 8)

// per-tile exclusive scan of accept counts: elocal[g] (within the tile), tile_sum[tile];
// one CTA per tile of the flattened tile space
__global__ void __launch_bounds__(512) k_scan_tiles(const uint8_t *__restrict__ amask, SegDev sg,
                                                    uint32_t *__restrict__ elocal, uint32_t *__restrict__ tile_sum) {
  __shared__ uint32_t wsum[16];
  const uint32_t T = blockIdx.x;
  const uint32_t st = seg_find(sg.toff, sg.nstreams, T);
  const uint64_t r0 = __ldg(sg.roff + st), R = __ldg(sg.roff + st + 1) - r0;
  const uint64_t base = (uint64_t)(T - __ldg(sg.toff + st)) * kScanTile + threadIdx.x * 8;
  uint32_t cnt[8], tot = 0;
  // whole runs at 8-byte aligned masks and 16-byte aligned prefixes (every refill range of a
  // uniform table in the 256-byte aligned scratch): one 8-byte load, two 16-byte stores
  const bool vec = base + 8 <= R && (reinterpret_cast<uintptr_t>(amask + r0 + base) & 7u) == 0 &&
                   (reinterpret_cast<uintptr_t>(elocal + r0 + base) & 15u) == 0;
  if (vec) {
    const uint2 m8 = __ldg(reinterpret_cast<const uint2 *>(amask + r0 + base));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      cnt[i] = __popc((m8.x >> (8 * i)) & 0xffu);
      cnt[4 + i] = __popc((m8.y >> (8 * i)) & 0xffu);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint64_t t = base + i;
      cnt[i] = t < R ? __popc(amask[r0 + t]) : 0u;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) tot += cnt[i];
  // block exclusive scan of per-thread totals
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < 16 ? wsum[lane] : 0u, si = s;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += v;
    }
    if (lane < 16) wsum[lane] = si - s;
    if (lane == 15) tile_sum[T] = si;
  }
  __syncthreads();
  uint32_t run = wsum[wid] + inc - tot;
  uint32_t ex[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    ex[i] = run;
    run += cnt[i];
  }
  if (vec) {
    uint4 *o = reinterpret_cast<uint4 *>(elocal + r0 + base);
    o[0] = make_uint4(ex[0], ex[1], ex[2], ex[3]);
    o[1] = make_uint4(ex[4], ex[5], ex[6], ex[7]);
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (base + i < R) elocal[r0 + base + i] = ex[i];
  }
}

// exclusive scan of the tile sums of each stream (one block per stream)
__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t *__restrict__ tile_sum, SegDev sg) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry;
  const uint32_t st = blockIdx.x;
  const uint32_t t0 = __ldg(sg.toff + st), tiles = __ldg(sg.toff + st + 1) - t0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < tiles; b0 += 1024) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t v = i < tiles ? tile_sum[t0 + i] : 0u;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      uint32_t s = wsum[lane], si = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= o) si += u;
      }
      wsum[lane] = si - s;
    }
    __syncthreads();
    const uint32_t excl = carry + wsum[wid] + inc - v;
    if (i < tiles) tile_sum[t0 + i] = excl;
    __syncthreads();
    if (threadIdx.x == 1023) carry = excl + v;
    __syncthreads();
  }
}

// exclusive prefix E(t) of stream st's accept counts, t in [0, R]
struct SegView {
  uint64_t r0;
  uint32_t R, t0;
};
__device__ __forceinline__ SegView seg_view(const SegDev &sg, uint32_t st) {
  SegView v;
  v.r0 = __ldg(sg.roff + st);
  v.R = (uint32_t)(__ldg(sg.roff + st + 1) - v.r0);
  v.t0 = __ldg(sg.toff + st);
  return v;
}
__device__ __forceinline__ uint32_t prefix_at(const uint32_t *elocal, const uint32_t *tile_off, const uint8_t *amask,
                                              const SegView &v, uint32_t t) {
  if (t < v.R) return elocal[v.r0 + t] + tile_off[v.t0 + t / kScanTile];
  const uint32_t l = v.R - 1;
  return elocal[v.r0 + l] + tile_off[v.t0 + l / kScanTile] + __popc(amask[v.r0 + l]);
}

// one warp per stream: call c starts at a fresh refill a_c; it ends at the first refill e
// whose inclusive prefix reaches E(a_c) + n; a_{c+1} = e + 1.  call_start of stream st:
// coff[st] + st .. coff[st+1] + st (calls + 1 entries; the last is the end of the last call).
__global__ void k_walk(const uint32_t *__restrict__ elocal, const uint32_t *__restrict__ tile_off,
                       const uint8_t *__restrict__ amask, SegDev sg, float mean_accept,
                       uint32_t *__restrict__ call_start, uint32_t *__restrict__ status) {
  const uint32_t st = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (st >= sg.nstreams) return;  // whole warps only
  const SegView v = seg_view(sg, st);
  const uint32_t n = __ldg(sg.n + st), calls = __ldg(sg.calls + st);
  const uint32_t guess = (uint32_t)((float)n / mean_accept);
  uint32_t *cs = call_start + __ldg(sg.coff + st) + st;
  uint32_t a = 0;
  bool bad = v.R == 0;
  uint32_t c = 0;
  // exclusive prefix at a, the start of the current call; afterwards it is carried over from
  // the search, where the lane that found a call's last refill e has read prefix_at(e + 1)
  uint32_t base = bad ? 0u : prefix_at(elocal, tile_off, amask, v, 0);
  for (; c < calls && !bad; ++c) {
    const uint32_t target = base + n;
    // smallest e >= a whose inclusive prefix reaches target (monotone in e), searched in
    // windows of 32 refills around the expected call length; `known` is a position already
    // seen to satisfy (its prefix in known_pv).  Upward moves stop at the refill range,
    // downward moves at a.
    uint32_t lo = a + (guess > 16 ? guess - 16 : 0);
    int64_t known = -1;
    uint32_t known_pv = 0, e = 0, next_base = 0;
    for (int it = 0;; ++it) {
      if (it > (1 << 22)) {  // cannot happen for a monotone prefix; bounded regardless
        bad = true;
        break;
      }
      const uint32_t j = lo + lane;
      const uint32_t pv = j < v.R ? prefix_at(elocal, tile_off, amask, v, j + 1) : 0u;
      const bool ok = (j < v.R) && pv >= target;
      const uint32_t bal = __ballot_sync(0xffffffffu, ok);
      if (bal == 0) {
        if (known >= 0) {
          e = (uint32_t)known;
          next_base = known_pv;
          break;
        }
        if (lo + 32 >= v.R) {
          bad = true;
          break;
        }
        lo += 32;
        continue;
      }
      const int first = __ffs(bal) - 1;
      const uint32_t first_pv = __shfl_sync(0xffffffffu, pv, first);
      if (first > 0 || lo == a) {
        e = lo + first;
        next_base = first_pv;
        break;
      }
      known = lo;
      known_pv = first_pv;
      lo = lo > a + 32 ? lo - 32 : a;
    }
    if (bad) break;
    if (lane == 0) cs[c] = a;
    a = e + 1;
    base = next_base;
  }
  if (lane == 0) {
    if (bad) atomicOr(status, kStatusRefillsExhausted);
    for (uint32_t r = bad ? c : calls; r <= calls; ++r) cs[r] = bad ? v.R : a;
  }
}

// Pointer doubling for the call starts (the same result as k_walk).  next(t) of stream s is
// the refill after a call that starts at refill t ends: e + 1 for the first e >= t whose
// inclusive prefix reaches E(t) + n, or R + 1 (absorbing) when the stream runs out; the start
// of call c is next applied c times to 0, assembled from the bits of c with the tables
// J_k = next^(2^k).
__global__ void k_next_start(const uint32_t *__restrict__ elocal, const uint32_t *__restrict__ tile_off,
                             const uint8_t *__restrict__ amask, SegDev sg, float mean_accept,
                             uint32_t *__restrict__ next) {
  const uint64_t total = __ldg(sg.roff + sg.nstreams);
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const uint32_t st = seg_find(sg.roff, sg.nstreams, g);
  const SegView v = seg_view(sg, st);
  const uint32_t t = (uint32_t)(g - v.r0), n = __ldg(sg.n + st);
  const uint32_t target = prefix_at(elocal, tile_off, amask, v, t) + n;
  // smallest e in [t, R) with E(e + 1) >= target; try the expected call length first
  uint32_t lo = t, hi = v.R;
  const uint32_t guess = t + 2u * (uint32_t)((float)n / mean_accept) + 64u;
  if (guess < v.R && prefix_at(elocal, tile_off, amask, v, guess + 1) >= target) hi = guess;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (prefix_at(elocal, tile_off, amask, v, mid + 1) >= target) hi = mid;
    else lo = mid + 1;
  }
  next[g] = lo < v.R ? lo + 1 : v.R + 1;
}

__global__ void k_next_square(const uint32_t *__restrict__ jin, uint32_t *__restrict__ jout, SegDev sg) {
  const uint64_t total = __ldg(sg.roff + sg.nstreams);
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const uint32_t st = seg_find(sg.roff, sg.nstreams, g);
  const uint64_t r0 = __ldg(sg.roff + st);
  const uint32_t R = (uint32_t)(__ldg(sg.roff + st + 1) - r0);
  const uint32_t a = jin[g];
  jout[g] = a < R ? jin[r0 + a] : R + 1;
}

// one thread per (stream, c), c = 0 .. calls: call_start[coff[s] + s + c]
__global__ void k_starts_from_tables(const uint32_t *__restrict__ tables, int levels, uint64_t refills, SegDev sg,
                                     uint32_t *__restrict__ call_start, uint32_t *__restrict__ status) {
  const uint64_t total = __ldg(sg.coff + sg.nstreams) + sg.nstreams;
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  uint32_t lo = 0, hi = sg.nstreams;  // stream s owns entries [coff[s] + s, coff[s+1] + s + 1)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(sg.coff + mid) + mid <= i) lo = mid;
    else hi = mid;
  }
  const uint32_t st = lo;
  const uint32_t c = (uint32_t)(i - (__ldg(sg.coff + st) + st));
  const uint64_t r0 = __ldg(sg.roff + st);
  const uint32_t R = (uint32_t)(__ldg(sg.roff + st + 1) - r0);
  uint32_t a = 0;
  for (int k = 0; k < levels; ++k)
    if ((c >> k) & 1u) a = a < R ? tables[(uint64_t)k * refills + r0 + a] : R + 1;
  call_start[i] = a <= R ? a : R;
  if (a > R && c == __ldg(sg.calls + st)) atomicOr(status, kStatusRefillsExhausted);
}

// ------------------------------------------------------------------ CPU mapping, phase 3

struct ModArgs {
  uint32_t q[3];
  uint64_t mu[3];   // floor(2^64 / q)
  uint32_t qr[3];   // floor(2^32 / q)
  uint32_t c32[3];  // 2^32 mod q
};

// (-1)^neg (hi 2^32 + lo) mod q_j for hi <= 1: lo mod q by one multiply-high (lo -
// floor(lo qr / 2^32) q is in [0, 2q)), plus 2^32 mod q when hi is set
__device__ __forceinline__ uint32_t residue_parts(uint32_t lo, uint32_t hi, uint32_t neg, const ModArgs &m, int j) {
  const uint32_t q = m.q[j];
  uint32_t r = mod_red1(lo - __umulhi(lo, m.qr[j]) * q, q);
  if (hi) r = mod_add(r, m.c32[j], q);
  return neg && r ? q - r : r;
}

// one CTA per call of the flattened call space: the accepted candidates of refills
// [a_c, a_{c+1}) in order, as residues out[ooff[st] + c * 3n ...][3][n].  Warp w of the CTA
// takes a contiguous run of the call's refills, 32 at a time: lane L loads the accept, bit-32
// and sign bits of refill t + L and, for k = 0..7, the low word of candidate L & 7 of refill
// t + 4k + L / 8 (eight coalesced 128-byte loads in flight per warp).  Per k the warp ballots the accepted lanes and packs
// them, in refill order and then candidate order (the order the reference consumes them), into
// a per-warp staging array; then every lane reduces one staged sample and the warp writes
// consecutive output positions.  Only the first position of each warp's run comes from the
// prefix tables.
constexpr int kScatterThreads = 256;
__global__ void __launch_bounds__(kScatterThreads)
    k_scatter(const uint32_t *__restrict__ cand_lo, const uint8_t *__restrict__ amask,
              const uint16_t *__restrict__ chs, const uint32_t *__restrict__ elocal,
              const uint32_t *__restrict__ tile_off, const uint32_t *__restrict__ call_start, SegDev sg, ModArgs m,
              uint32_t *__restrict__ out) {
  __shared__ uint2 stage[kScatterThreads / 32][256];
  const uint32_t st = seg_find(sg.coff, sg.nstreams, blockIdx.x);
  const uint64_t cs0 = __ldg(sg.coff + st);
  const uint32_t c = (uint32_t)(blockIdx.x - cs0);
  const SegView v = seg_view(sg, st);
  const uint32_t n = __ldg(sg.n + st);
  const uint32_t *cs = call_start + cs0 + st;
  const uint32_t a = cs[c], b = min(cs[c + 1], v.R);
  if (a >= b) return;
  const uint32_t lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
  const uint32_t span = ((b - a + nw - 1) / nw + 3u) & ~3u;  // refills per warp
  const uint32_t t0 = a + (threadIdx.x >> 5) * span;
  if (t0 >= b) return;  // whole warps leave together; no CTA barrier follows
  const uint32_t t1 = min(t0 + span, b);
  uint32_t pos = prefix_at(elocal, tile_off, amask, v, t0) - prefix_at(elocal, tile_off, amask, v, a);
  uint32_t *o = out + __ldg(sg.ooff + st) + (size_t)c * 3 * n;
  uint2 *sw = stage[threadIdx.x >> 5];
  const uint32_t below = (1u << lane) - 1u, ci = lane & 7u;
  for (uint32_t t = t0; t < t1 && pos < n; t += 32) {
    // refill t + lane: accept bits, bit 32 of each |value| (<< 8), signs (<< 16)
    const uint32_t mk = t + lane < t1 ? (uint32_t)__ldg(amask + v.r0 + t + lane) |
                                            ((uint32_t)__ldg(chs + v.r0 + t + lane) << 8)
                                      : 0u;
    uint32_t lv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t r = t + 4 * k + (lane >> 3);
      lv[k] = r < t1 ? __ldg(cand_lo + (v.r0 + r) * 8 + ci) : 0u;
    }
    uint32_t cnt = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t meta = __shfl_sync(0xffffffffu, mk, 4 * k + (lane >> 3)) >> ci;
      const bool acc = meta & 1u;
      const uint32_t bal = __ballot_sync(0xffffffffu, acc);
      if (acc)  // staged as (low word, bit 32 | sign << 31)
        sw[cnt + __popc(bal & below)] = make_uint2(lv[k], ((meta >> 8) & 1u) | (((meta >> 16) & 1u) << 31));
      cnt += __popc(bal);
    }
    __syncwarp();
    for (uint32_t i = lane; i < cnt && pos + i < n; i += 32) {
      const uint2 sv = sw[i];
#pragma unroll
      for (int j = 0; j < 3; ++j) o[j * n + pos + i] = residue_parts(sv.x, sv.y & 1u, sv.y >> 31, m, j);
    }
    __syncwarp();  // the next step overwrites the staging array
    pos += cnt;
  }
}

// segment table of nstreams equal streams (calls x n each, refills R each, output stride
// `ostride` words per stream)
__global__ void k_seg_uniform(uint32_t nstreams, uint32_t calls, uint32_t n, uint32_t R, uint32_t tiles,
                              uint64_t ostride, uint32_t *__restrict__ sn, uint32_t *__restrict__ scalls,
                              uint64_t *__restrict__ roff, uint32_t *__restrict__ toff, uint64_t *__restrict__ coff,
                              uint64_t *__restrict__ ooff) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nstreams) return;
  roff[i] = (uint64_t)i * R;
  toff[i] = i * tiles;
  coff[i] = (uint64_t)i * calls;
  if (i < nstreams) {
    sn[i] = n;
    scalls[i] = calls;
    ooff[i] = (uint64_t)i * ostride;
  }
}

// ------------------------------------------------------------------ GPU mapping

// chained AES refill of the GPU mapping (src/AES.cuh:380-435): 18 blocks (bytes 0..287)
// into buf; blocks 18..23 only when a uniform draw needs them.
__device__ __forceinline__ void chain_blocks(uint32_t *buf, int from, int to, uint32_t &s0, uint32_t &s1,
                                             uint32_t &s2, uint32_t &s3, const uint32_t (&rk)[60],
                                             const AesCtx &c) {
  for (int m = from; m < to; ++m) {
    aes256_rounds(s0, s1, s2, s3, rk, c);
    buf[4 * m] = s0;
    buf[4 * m + 1] = s1;
    buf[4 * m + 2] = s2;
    buf[4 * m + 3] = s3;
  }
}

// 512 threads: the 128 KB of tables allow one CTA per SM, and the chained blocks leave one
// thread little independent work, so the CTA brings as many warps as the register file holds
constexpr int kGpuMapThreads = 512;
template <int SIG>
__global__ void __launch_bounds__(kGpuMapThreads, 1)
    k_gauss_gpu_map(const uint32_t *__restrict__ rkey, uint32_t poly0, uint32_t npolys, uint32_t n, double kinv,
                    ModArgs m, uint32_t *__restrict__ out, uint32_t *__restrict__ status) {
  extern __shared__ __align__(128) uint8_t smem[];
  aes_fill_tables(smem);
  __syncthreads();
  const AesCtx c{smem, (threadIdx.x & 31u) * 4u};
  uint32_t rk[60];
#pragma unroll
  for (int i = 0; i < 60; ++i) rk[i] = __ldg(rkey + i);
  const uint32_t T = n / 8;
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= npolys * T) return;
  const uint32_t p = gid / T, t = gid - p * T, poly = poly0 + p;
  uint32_t buf[96];
  uint32_t y[8], x[8], acc = 0, k8 = 0;
  uint64_t z[8];
  uint32_t i = 8, rep = 0;
  uint32_t *o = out + (size_t)p * 3 * n;
  bool gave_up = false;
  for (uint32_t j = 0; j < 8 && !gave_up; ++j) {
    uint32_t k = 0;
    for (;;) {
      if (i == 8) {
        if (rep >= kMaxRefillsPerThread) {  // never reached by a working sampler; bounded anyway
          atomicOr(status, kStatusRefillCap);
          gave_up = true;
          break;
        }
        const uint32_t ctr = poly * 5u * T * 24u + rep * T * 24u + t * 24u;
        uint32_t s0 = rk[0], s1 = rk[1], s2 = rk[2], s3 = ctr ^ rk[3];
        aes256_rounds(s0, s1, s2, s3, rk, c);
        buf[0] = s0; buf[1] = s1; buf[2] = s2; buf[3] = s3;
        chain_blocks(buf, 1, 18, s0, s1, s2, s3, rk, c);
        int have = 18;
        // uniform words from byte 200 (word 50)
        int w = 0;
        for (int jj = 0; jj < 8; ++jj) {
          uint32_t xx;
          for (;;) {
            const int wi = 50 + w;
            if (wi >= 96) {
              atomicOr(status, kStatusUniformOverrun);
              xx = 0;
              break;
            }
            if ((wi >> 2) >= have) {
              chain_blocks(buf, have, have + 1, s0, s1, s2, s3, rk, c);
              ++have;
            }
            xx = bswap32(buf[wi]);
            ++w;
            if (uniform_ok<SIG>(xx)) break;
          }
          y[jj] = uniform_reduce<SIG>(xx);
        }
        for (int h = 0; h < 2; ++h) {
          const int bw = 25 * h;  // word offset of r + 100*h
          for (int ln = 0; ln < 4; ++ln) {
            const uint64_t r2 = ((uint64_t)bswap32(buf[bw + 8 + 2 * ln])) |
                                ((uint64_t)bswap32(buf[bw + 9 + 2 * ln]) << 32);
            x[4 * h + ln] = cdt_sample<false>(r2, 0);
          }
        }
        k8 = buf[70] >> 24;  // byte 280
        acc = 0;
        for (int h = 0; h < 2; ++h) {
          const int bw = 25 * h;
          const uint32_t ew = buf[bw + 24];  // bytes 96..99 (+100 h)
          for (int ln = 0; ln < 4; ++ln) {
            const uint64_t rm = ((uint64_t)bswap32(buf[bw + 16 + 2 * ln])) |
                                ((uint64_t)bswap32(buf[bw + 17 + 2 * ln]) << 32);
            const uint32_t rexp = (ew >> (24 - 8 * ln)) & 0xffu;
            uint64_t zz;
            const bool b = candidate<SIG, 2>(x[4 * h + ln], y[4 * h + ln], rm, rexp, kinv, zz);
            z[4 * h + ln] = zz;
            acc |= (uint32_t)b << (4 * h + ln);
          }
        }
        i = 0;
        ++rep;
      }
      k = (k8 >> i) & 1u;
      ++i;
      if (accept_final((acc >> (i - 1)) & 1u, z[i - 1], k)) break;
    }
    if (gave_up) break;
    const uint64_t zs = z[i - 1];  // K x + y < 8K < 2^33
    if (zs >> 33) atomicOr(status, kStatusWideSample);
    const uint32_t pos = 8 * t + j;
#pragma unroll
    for (int jj = 0; jj < 3; ++jj)
      o[jj * n + pos] = residue_parts((uint32_t)zs, (uint32_t)(zs >> 32) & 1u, k, m, jj);
  }
}

// ------------------------------------------------------------------ uniform a

// sample_polya (src/sample.c:56-128): AES-CTR (nonce 0) bytes, a_i = le64(bytes 8i..8i+7) mod q_j
__global__ void __launch_bounds__(256) k_polya(const uint32_t *__restrict__ rkey, uint32_t n, ModArgs m,
                                               uint32_t *__restrict__ a) {
  extern __shared__ __align__(128) uint8_t smem[];
  aes_fill_tables(smem);
  __syncthreads();
  const AesCtx c{smem, (threadIdx.x & 31u) * 4u};
  uint32_t rk[60];
#pragma unroll
  for (int i = 0; i < 60; ++i) rk[i] = __ldg(rkey + i);
  const uint32_t blk = blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= n / 2) return;
  uint32_t W[4];
  aes256_ctr_block(W, 0u, blk, rk, c);
  const uint64_t v0 = le64_of(W[0], W[1]), v1 = le64_of(W[2], W[3]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    a[j * n + 2 * blk] = mod_u64(v0, m.mu[j], m.q[j]);
    a[j * n + 2 * blk + 1] = mod_u64(v1, m.mu[j], m.q[j]);
  }
}

}  // namespace

// ------------------------------------------------------------------ host side


static ModArgs mod_args() {
  ModArgs m;
  for (int j = 0; j < 3; ++j) {
    m.q[j] = kRefPrimes[j];
    unsigned __int128 one = (unsigned __int128)1 << 64;
    m.mu[j] = (uint64_t)(one / kRefPrimes[j]);
    m.qr[j] = (uint32_t)((1ull << 32) / kRefPrimes[j]);
    m.c32[j] = (uint32_t)((1ull << 32) % kRefPrimes[j]);
  }
  return m;
}

static double kinv_of(int sig) {
  const uint64_t K = sigma_k(sig);
  return -1.0 / (double)(int64_t)(K * K);
}

static uint8_t gmul8(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  while (b) {
    if (b & 1) r ^= a;
    a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
    b >>= 1;
  }
  return r;
}

void aes_key_expand(const uint8_t key[32], uint32_t w[60]) {
  static uint8_t sbox[256];
  static bool ready = false;
  if (!ready) aes_sbox(sbox), ready = true;
  uint8_t rc = 1;
  for (int i = 0; i < 8; ++i)
    w[i] = ((uint32_t)key[4 * i] << 24) | ((uint32_t)key[4 * i + 1] << 16) | ((uint32_t)key[4 * i + 2] << 8) |
           key[4 * i + 3];
  for (int i = 8; i < 60; ++i) {
    uint32_t t = w[i - 1];
    auto sub = [&](uint32_t v) {
      return ((uint32_t)sbox[v >> 24] << 24) | ((uint32_t)sbox[(v >> 16) & 255] << 16) |
             ((uint32_t)sbox[(v >> 8) & 255] << 8) | sbox[v & 255];
    };
    if (i % 8 == 0) {
      t = sub((t << 8) | (t >> 24)) ^ ((uint32_t)rc << 24);
      rc = gmul8(rc, 2);
    } else if (i % 8 == 4) {
      t = sub(t);
    }
    w[i] = w[i - 8] ^ t;
  }
}

void aes_sbox(uint8_t out[256]) {
  // FIPS-197 5.1.1: multiplicative inverse in GF(2^8) followed by the affine map
  for (int x = 0; x < 256; ++x) {
    uint8_t inv = 0;
    if (x)
      for (int y = 1; y < 256; ++y)
        if (gmul8((uint8_t)x, (uint8_t)y) == 1) {
          inv = (uint8_t)y;
          break;
        }
    uint8_t s = inv;
    for (int r = 1; r <= 4; ++r) s ^= (uint8_t)((inv << r) | (inv >> (8 - r)));
    out[x] = s ^ 0x63;
  }
}

// AES-256 key expansion (FIPS-197 5.2) on the device, one key per thread, into the
// big-endian round-key words of aes_key_expand: rk[i][60] from seeds[perm ? perm[i] : i][32]
__global__ void k_expand_keys(const uint8_t *__restrict__ seeds, const uint32_t *__restrict__ perm, uint32_t count,
                              uint32_t *__restrict__ rk) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint8_t *k = seeds + 32 * (size_t)(perm ? perm[i] : i);
  uint32_t w[60];
#pragma unroll
  for (int j = 0; j < 8; ++j)
    w[j] = ((uint32_t)k[4 * j] << 24) | ((uint32_t)k[4 * j + 1] << 16) | ((uint32_t)k[4 * j + 2] << 8) | k[4 * j + 3];
#pragma unroll
  for (int j = 8; j < 60; ++j) {
    uint32_t t = w[j - 1];
    if (j % 8 == 0) t = (t << 8) | (t >> 24);
    if (j % 8 == 0 || j % 8 == 4)
      t = ((uint32_t)c_sbox[t >> 24] << 24) | ((uint32_t)c_sbox[(t >> 16) & 255] << 16) |
          ((uint32_t)c_sbox[(t >> 8) & 255] << 8) | c_sbox[t & 255];
    if (j % 8 == 0) t ^= (1u << (j / 8 - 1)) << 24;  // round constants 1, 2, 4, ..., 64
    w[j] = w[j - 8] ^ t;
  }
  uint32_t *o = rk + (size_t)i * 60;
#pragma unroll
  for (int j = 0; j < 60; ++j) o[j] = w[j];
}

int expand_keys_device(const uint8_t *d_seeds, const uint32_t *d_perm, uint32_t count, uint32_t *d_rk,
                       cudaStream_t s) {
  if (!count) return CUFE_OK;
  note_launch(), k_expand_keys<<<(count + 127) / 128, 128, 0, s>>>(d_seeds, d_perm, count, d_rk);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

int sampler_init_device() {
  uint8_t sbox[256];
  aes_sbox(sbox);
  CUFE_CUDA(cudaMemcpyToSymbol(c_sbox, sbox, 256));
  CUFE_CUDA(cudaFuncSetAttribute(k_cand_cpu<0, false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  CUFE_CUDA(cudaFuncSetAttribute(k_cand_cpu<1, false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  CUFE_CUDA(cudaFuncSetAttribute(k_cand_cpu<2, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  CUFE_CUDA(cudaFuncSetAttribute(k_gauss_gpu_map<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  CUFE_CUDA(cudaFuncSetAttribute(k_gauss_gpu_map<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  CUFE_CUDA(cudaFuncSetAttribute(k_gauss_gpu_map<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  CUFE_CUDA(cudaFuncSetAttribute(k_polya, cudaFuncAttributeMaxDynamicSharedMemorySize, kAesSmemBytes));
  return CUFE_OK;
}

// Accepted candidates per 8-candidate refill of the CPU mapping, measured on the oracle over
// 4 M AES-CTR refills per sigma: mean 5.4436 / 4.3942 / 3.0948 (+-0.0007) and variance 1.74 /
// 1.98 / 1.90 for S1 / S2 / S3 (the uint32 truncation of src/gauss.c:849 rejects more at large
// K).  The means below are those rounded down, the variance bound is 2.0 for all three.
static double mean_accept(int sig) { return sig == 0 ? 5.443 : (sig == 1 ? 4.393 : 3.094); }
constexpr double kAcceptVarBound = 2.0;

// Refills precomputed for `calls` consecutive calls of n samples.  A call consumes r refills,
// the first whose accepted total reaches n; E[r] = (n + overshoot) / mu < n / mu + 1 (the
// overshoot averages below 1.4 samples), and over many calls sum(r) has variance about
// calls n v / mu^3 (renewal count).  The range is calls (n / mu + 1) plus 12 of those
// standard deviations plus 64.  Against the exact distribution of r (dynamic programming
// over the measured accept-count histogram), that is at least 13 standard deviations of
// sum(r) above its mean for every n in 16..8192 and 1..4096 calls, and 0.2-0.6% above the
// mean need for long streams (the former 3% margin over rounded-down means was 6%).  A
// stream that still ran short sets kStatusRefillsExhausted (checked by the host) and never
// reads past its range.
uint32_t cpu_map_refills(uint32_t calls, uint32_t n, int sig) {
  const double mu = mean_accept(sig), cn = (double)calls * (double)n;
  const double need = (double)calls * ((double)n / mu + 1.0);
  const double sd = std::sqrt(cn * kAcceptVarBound / (mu * mu * mu));
  const uint32_t R = (uint32_t)std::ceil(need + 12.0 * sd) + 64;
  return (R + 31) & ~31u;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

SegLayout seg_layout(uint32_t S) {
  SegLayout L;
  size_t o = 0;
  L.n = o;
  o += align256((size_t)S * 4);
  L.calls = o;
  o += align256((size_t)S * 4);
  L.toff = o;
  o += align256((size_t)(S + 1) * 4);
  L.roff = o;
  o += align256((size_t)(S + 1) * 8);
  L.coff = o;
  o += align256((size_t)(S + 1) * 8);
  L.ooff = o;
  o += align256((size_t)S * 8);
  L.bytes = o;
  return L;
}

SegDev seg_bind(void *base, uint32_t S) {
  const SegLayout L = seg_layout(S);
  uint8_t *b = static_cast<uint8_t *>(base);
  SegDev d;
  d.nstreams = S;
  d.n = reinterpret_cast<const uint32_t *>(b + L.n);
  d.calls = reinterpret_cast<const uint32_t *>(b + L.calls);
  d.toff = reinterpret_cast<const uint32_t *>(b + L.toff);
  d.roff = reinterpret_cast<const uint64_t *>(b + L.roff);
  d.coff = reinterpret_cast<const uint64_t *>(b + L.coff);
  d.ooff = reinterpret_cast<const uint64_t *>(b + L.ooff);
  return d;
}

SegSizes seg_fill_host(int sig, uint32_t S, const uint32_t *calls, const uint32_t *n, const uint64_t *ooff,
                       void *host_base) {
  const SegLayout L = seg_layout(S);
  uint8_t *b = static_cast<uint8_t *>(host_base);
  uint32_t *hn = reinterpret_cast<uint32_t *>(b + L.n), *hc = reinterpret_cast<uint32_t *>(b + L.calls);
  uint32_t *ht = reinterpret_cast<uint32_t *>(b + L.toff);
  uint64_t *hr = reinterpret_cast<uint64_t *>(b + L.roff), *hco = reinterpret_cast<uint64_t *>(b + L.coff);
  uint64_t *ho = reinterpret_cast<uint64_t *>(b + L.ooff);
  SegSizes z{S, 0, 0, 0, 0, false};
  for (uint32_t i = 0; i < S; ++i) {
    const uint32_t R = cpu_map_refills(calls[i], n[i], sig);
    hn[i] = n[i];
    hc[i] = calls[i];
    ho[i] = ooff ? ooff[i] : 0;
    hr[i] = z.refills;
    ht[i] = z.tiles;
    hco[i] = z.calls;
    z.refills += R;
    z.tiles += (R + kScanTile - 1) / kScanTile;
    z.calls += calls[i];
    z.max_calls = std::max(z.max_calls, calls[i]);
  }
  hr[S] = z.refills;
  ht[S] = z.tiles;
  hco[S] = z.calls;
  z.doubling = seg_auto_doubling(z.refills, z.max_calls);
  return z;
}

static SegSizes seg_uniform_sizes(uint32_t S, uint32_t calls, uint32_t n, int sig) {
  const uint32_t R = cpu_map_refills(calls, n, sig);
  return SegSizes{S, (uint64_t)S * R, S * ((R + kScanTile - 1) / kScanTile), (uint64_t)S * calls, calls,
                  seg_auto_doubling((uint64_t)S * R, calls)};
}

static int g_call_search = 0;
void set_call_search(int mode) { g_call_search = mode; }
int get_call_search() { return g_call_search; }

constexpr uint64_t kDoublingMaxRefills = (uint64_t)32 << 20;

static int doubling_levels(uint32_t max_calls) {
  int k = 1;
  while (k < 31 && (1u << k) <= max_calls) ++k;
  return k;  // bit_length(max_calls), at least 1
}
// Doubling costs about 6.4 ps per refill per table level (memory-bound gathers); the walk
// about 1.0-1.4 us per call of its longest stream (serial dependent loads), both measured on
// a B200 (sigma_3 at n = 4096, l = 784: doubling 0.48 / 1.12 ms at 8 / 16 encryptions, walk
// 0.78 ms up to 16 and 1.13 ms from 24).  Doubling is chosen when it is the cheaper of the two
// and its tables stay below 32 Mi refills.
bool seg_auto_doubling(uint64_t refills, uint32_t max_calls) {
  if (g_call_search == 1 || refills > kDoublingMaxRefills) return false;
  if (g_call_search == 2) return true;
  return refills * (uint64_t)doubling_levels(max_calls) <= (uint64_t)max_calls * 200000u;
}

size_t seg_scratch_bytes(const SegSizes &z) {
  size_t b = align256(z.refills * 32) + align256(z.refills) + align256(z.refills * 2) + align256(z.refills * 4) +
             align256((size_t)z.tiles * 4) +
             align256((z.calls + z.nstreams) * 4);
  if (z.doubling) b += (size_t)doubling_levels(z.max_calls) * align256(z.refills * 4);
  return b;
}

size_t cpu_map_workspace_bytes(uint32_t nstreams, uint32_t calls, uint32_t n, int sig) {
  return seg_layout(nstreams).bytes + seg_scratch_bytes(seg_uniform_sizes(nstreams, calls, n, sig));
}

int sample_cpu_map_seg(int sig, const SegDev &sg, const SegSizes &z, const uint32_t *d_rkeys, uint32_t *d_out,
                       void *scratch, uint32_t *d_status, int num_sms, cudaStream_t s) {
  if (sig < 0 || sig > 2 || z.nstreams == 0 || z.tiles >= (1u << 31) || z.calls >= (1ull << 31) ||
      z.refills >= (1ull << 32) - (1ull << 24))
    return CUFE_ERR_INVALID;
  uint8_t *p = static_cast<uint8_t *>(scratch);
  auto take = [&](size_t x) {
    uint8_t *r = p;
    p += align256(x);
    return r;
  };
  uint32_t *cand = reinterpret_cast<uint32_t *>(take(z.refills * 32));  // low words of |candidate|
  uint8_t *amask = take(z.refills);
  uint16_t *chs = reinterpret_cast<uint16_t *>(take(z.refills * 2));  // bit 32 of each, signs << 8
  uint32_t *elocal = reinterpret_cast<uint32_t *>(take(z.refills * 4));
  uint32_t *tsum = reinterpret_cast<uint32_t *>(take((size_t)z.tiles * 4));
  uint32_t *cstart = reinterpret_cast<uint32_t *>(take((z.calls + z.nstreams) * 4));
  const double kinv = kinv_of(sig);
  const uint32_t grid =
      (uint32_t)std::min<uint64_t>((uint64_t)num_sms, (z.refills + kCandThreads - 1) / kCandThreads);
  if (grid > 0) {
    ProfScope ps(sig == 0 ? "sample_cand_s1" : (sig == 1 ? "sample_cand_s2" : "sample_cand_s3"), s);
    if (sig == 0)
      note_launch(), k_cand_cpu<0, false, 0><<<grid, kCandThreads, kAesSmemBytes, s>>>(d_rkeys, sg, kinv, cand, amask, chs,
                                                                             d_status);
    else if (sig == 1)
      note_launch(), k_cand_cpu<1, false, 0><<<grid, kCandThreads, kAesSmemBytes, s>>>(d_rkeys, sg, kinv, cand, amask, chs,
                                                                             d_status);
    else
      note_launch(), k_cand_cpu<2, true, 1><<<grid, kCandThreads, kAesSmemBytes, s>>>(d_rkeys, sg, kinv, cand, amask, chs,
                                                                             d_status);
  }
  CUFE_CUDA(cudaGetLastError());
  if (z.tiles) {
    ProfScope ps("sample_scan", s);
    note_launch(), k_scan_tiles<<<z.tiles, 512, 0, s>>>(amask, sg, elocal, tsum);
    note_launch(), k_scan_sums<<<z.nstreams, 1024, 0, s>>>(tsum, sg);
  }
  if (z.doubling) {
    const int levels = doubling_levels(z.max_calls);
    uint32_t *tab = reinterpret_cast<uint32_t *>(take((size_t)levels * align256(z.refills * 4)));
    const uint64_t stride = align256(z.refills * 4) / 4;
    ProfScope ps("sample_walk", s);
    const unsigned rg = (unsigned)((z.refills + 255) / 256);
    note_launch(), k_next_start<<<rg, 256, 0, s>>>(elocal, tsum, amask, sg, (float)mean_accept(sig), tab);
    for (int k = 1; k < levels; ++k) note_launch(), k_next_square<<<rg, 256, 0, s>>>(tab + (k - 1) * stride, tab + k * stride, sg);
    note_launch(), k_starts_from_tables<<<(unsigned)((z.calls + z.nstreams + 255) / 256), 256, 0, s>>>(tab, levels, stride, sg,
                                                                                        cstart, d_status);
  } else {
    ProfScope ps("sample_walk", s);
    note_launch(), k_walk<<<(z.nstreams + 3) / 4, 128, 0, s>>>(elocal, tsum, amask, sg, (float)mean_accept(sig), cstart, d_status);
  }
  CUFE_CUDA(cudaGetLastError());
  if (d_out && z.calls) {
    ProfScope ps_sc("sample_scatter", s);
    note_launch(), k_scatter<<<(uint32_t)z.calls, kScatterThreads, 0, s>>>(cand, amask, chs, elocal, tsum, cstart, sg,
                                                                           mod_args(), d_out);
    CUFE_CUDA(cudaGetLastError());
  }
  return CUFE_OK;
}

// the uniform case: nstreams equal streams, tables built on the device (capturable)
static int seg_uniform(uint32_t nstreams, uint32_t calls, uint32_t n, int sig, void *ws, cudaStream_t s, SegDev *sg,
                       SegSizes *z, void **scratch) {
  const SegLayout L = seg_layout(nstreams);
  *z = seg_uniform_sizes(nstreams, calls, n, sig);
  if (z->refills / nstreams >= (1ull << 32) / 24) return CUFE_ERR_INVALID;  // AES counter range
  uint8_t *b = static_cast<uint8_t *>(ws);
  *sg = seg_bind(b, nstreams);
  const uint32_t R = (uint32_t)(z->refills / nstreams);
  note_launch(), k_seg_uniform<<<(nstreams + 256) / 256, 256, 0, s>>>(
      nstreams, calls, n, R, z->tiles / nstreams, (uint64_t)calls * 3 * n, reinterpret_cast<uint32_t *>(b + L.n),
      reinterpret_cast<uint32_t *>(b + L.calls), reinterpret_cast<uint64_t *>(b + L.roff),
      reinterpret_cast<uint32_t *>(b + L.toff), reinterpret_cast<uint64_t *>(b + L.coff),
      reinterpret_cast<uint64_t *>(b + L.ooff));
  CUFE_CUDA(cudaGetLastError());
  *scratch = b + L.bytes;
  return CUFE_OK;
}

int sample_cpu_map(int sig, uint32_t nstreams, const uint32_t *d_rkeys, uint32_t calls, uint32_t n,
                   uint32_t *d_out, void *ws, uint32_t *d_status, int num_sms, cudaStream_t s) {
  SegDev sg;
  SegSizes z;
  void *scratch;
  int rc = seg_uniform(nstreams, calls, n, sig, ws, s, &sg, &z, &scratch);
  if (rc) return rc;
  return sample_cpu_map_seg(sig, sg, z, d_rkeys, d_out, scratch, d_status, num_sms, s);
}

int sample_gpu_map(int sig, const uint32_t *d_rkey, uint32_t poly0, uint32_t npolys, uint32_t n, uint32_t *d_out,
                   uint32_t *d_status, cudaStream_t s) {
  const uint32_t threads = npolys * (n / 8);
  const uint32_t grid = (threads + kGpuMapThreads - 1) / kGpuMapThreads;
  const double kinv = kinv_of(sig);
  ProfScope ps("sample_gpu_map", s);
  if (sig == 0)
    note_launch(), k_gauss_gpu_map<0><<<grid, kGpuMapThreads, kAesSmemBytes, s>>>(d_rkey, poly0, npolys, n, kinv,
                                                                               mod_args(), d_out, d_status);
  else if (sig == 1)
    note_launch(), k_gauss_gpu_map<1><<<grid, kGpuMapThreads, kAesSmemBytes, s>>>(d_rkey, poly0, npolys, n, kinv,
                                                                               mod_args(), d_out, d_status);
  else
    note_launch(), k_gauss_gpu_map<2><<<grid, kGpuMapThreads, kAesSmemBytes, s>>>(d_rkey, poly0, npolys, n, kinv,
                                                                               mod_args(), d_out, d_status);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

int sample_polya(const uint32_t *d_rkey, uint32_t n, uint32_t *d_a, cudaStream_t s) {
  const uint32_t grid = (n / 2 + 255) / 256;
  ProfScope ps("sample_polya", s);
  note_launch(), k_polya<<<grid, 256, kAesSmemBytes, s>>>(d_rkey, n, mod_args(), d_a);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

}  // namespace cufe
