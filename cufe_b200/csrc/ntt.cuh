// ntt.cuh -- negacyclic NTT / INTT cores for one residue polynomial per thread group.
//
// Transform (reference: src/ntt.c:38-114): forward Cooley-Tukey with the psi powers
// merged (natural order in, bit-reversed order out), inverse Gentleman-Sande (bit-reversed
// in, natural out) including the factor n^-1.  Any exact implementation of this linear map
// gives the reference's values after canonical reduction, so the loop order is free.
//
// B200 design: n/E threads per residue polynomial, E = 2^LE coefficients per thread held in
// registers (E = 16 everywhere; the batched transform kernel also has E = 32 and 64 forms,
// picked by the ring's tuner).  The log2(n) butterfly stages are grouped into passes of up
// to LE stages (radix E); a pass touches only the E coefficients of a thread, and consecutive passes
// exchange coefficients through shared memory (one __syncthreads per exchange), one padding
// word per 32 (64 for radix 64) and, in the middle radix-16 pass, thread bits 4 and 5
// swapped: every exchange pattern of these plans is free of bank conflicts (n >= 1024) and
// every address is a per-thread base plus an immediate.  The smaller pass
// (log2(n) mod LE stages) comes first so that the strided passes are the early ones, whose
// warps touch 32 consecutive words.  Twiddles use Shoup's precomputed quotient (1 mul.hi +
// 2 mul.lo per product) and residues stay canonical in [0, q), q < 2^31, between kernels.
// The inverse folds n^-1 into its last stage.
#pragma once
#include "cufe_internal.cuh"

namespace cufe {

template <int LOGN, int LE = 4>
struct NttPlan {
  static constexpr int E = 1 << LE;  // coefficients per thread (radix of the full passes)
  static constexpr int N = 1 << LOGN;
  static constexpr int T = N / E;  // threads per residue polynomial
  static constexpr int NP = (LOGN + LE - 1) / LE;
  static constexpr int R0 = LOGN - LE * (NP - 1);
  // shared-memory layout of an exchange: coefficient j at word pad(j) = j + (j >> PADS), one
  // padding word per 2^PADS.  pad is additive over disjoint bits, so a thread's address of
  // register e is pad(idx_th) + pad(idx_e): a per-thread base plus an immediate offset.
  static constexpr int PADS = LE == 6 ? 6 : 5;
  static constexpr int SMEM_WORDS = N + (N >> PADS);
  __host__ __device__ static constexpr int pad(int j) { return j + (j >> PADS); }
  __host__ __device__ static constexpr int radix_bits(int p) { return p == 0 ? R0 : LE; }
  __host__ __device__ static constexpr int first_stage(int p) { return p == 0 ? 0 : R0 + LE * (p - 1); }
  // A radix-16 pass whose warp lanes would cover index bits 0..3 and 8 (the middle passes:
  // thread bits below position 4, the rest above the pass's 4 register bits) takes thread
  // bit 5 in place of bit 4, so its fifth lane bit lands on index bit 9, whose padded weight
  // (512 + 16) completes the bank set of bits 0..3; every exchange is then conflict-free.
  __host__ __device__ static constexpr bool lane_swap(int p) {
    return LE == 4 && LOGN - first_stage(p) - radix_bits(p) == 4 && T >= 64;
  }
  template <int PASS>
  __host__ __device__ static constexpr int vth(int th) {
    return lane_swap(PASS) ? ((th & ~0x30) | ((th >> 1) & 0x10) | ((th << 1) & 0x20)) : th;
  }
  // coefficient index held in register e by thread th during pass PASS.  The bits that come
  // from th and the bits that come from e are disjoint, so idx = idx_th(th) + idx_e(e), the
  // second a compile-time constant (an immediate offset in every load and store).  A pass
  // of rb < LE stages runs E >> rb butterfly blocks per thread ("virtual threads" v*T + th).
  template <int PASS>
  __host__ __device__ static constexpr int idx_th(int th) {
    constexpr int rb = radix_bits(PASS), s0 = first_stage(PASS);
    constexpr int plo = LOGN - s0 - rb, phi = LOGN - 1 - s0;
    const int t = vth<PASS>(th);
    return ((t >> plo) << (phi + 1)) | (t & ((1 << plo) - 1));
  }
  template <int PASS>
  __host__ __device__ static constexpr int idx_e(int e) {
    constexpr int rb = radix_bits(PASS), s0 = first_stage(PASS);
    constexpr int plo = LOGN - s0 - rb, phi = LOGN - 1 - s0;
    return ((((e >> rb) * T) >> plo) << (phi + 1)) | ((e & ((1 << rb) - 1)) << plo) | (((e >> rb) * T) & ((1 << plo) - 1));
  }
  template <int PASS>
  __device__ __forceinline__ static int idx(int th, int e) {
    return idx_th<PASS>(th) + idx_e<PASS>(e);
  }
  static_assert(pad(N - 1) < SMEM_WORDS, "exchange layout");
};

// P residue polynomials per thread group (same modulus, shared twiddles and addresses):
// polynomial p uses registers a[p][] and shared words sm[p * SMEM_WORDS ...]; every address is
// one per-thread base plus a compile-time offset (pad is additive over the disjoint bits of
// idx_th and idx_e).
template <int LOGN, int FROM, int TO, int P_, int LE, int E>
__device__ __forceinline__ void ntt_exchange(uint32_t (&a)[P_][E], uint32_t *sm, int th) {
  using P = NttPlan<LOGN, LE>;
  uint32_t *wb = sm + P::pad(P::template idx_th<FROM>(th));
#pragma unroll
  for (int e = 0; e < E; ++e) {
#pragma unroll
    for (int p = 0; p < P_; ++p) wb[p * P::SMEM_WORDS + P::pad(P::template idx_e<FROM>(e))] = a[p][e];
  }
  __syncthreads();
  const uint32_t *rb = sm + P::pad(P::template idx_th<TO>(th));
#pragma unroll
  for (int e = 0; e < E; ++e) {
#pragma unroll
    for (int p = 0; p < P_; ++p) a[p][e] = rb[p * P::SMEM_WORDS + P::pad(P::template idx_e<TO>(e))];
  }
}

// moduli below this take the small-modulus butterflies (SQ) where a kernel offers them
constexpr uint32_t kSmallQ = 1u << 27;

struct InvScale {
  uint32_t ninv, ninv_sh, w1n, w1n_sh;
};

// twiddles (w, w_shoup) tw[ti0 .. ti0+NG-1]: pairs of entries per 16-byte load when NG >= 2
// (ti0 is then even, so the load is aligned)
template <int NG>
__device__ __forceinline__ void load_twiddles(const uint2 *__restrict__ tw, int ti0, uint32_t (&w)[NG],
                                              uint32_t (&wsh)[NG]) {
  if constexpr (NG == 1) {
    const uint2 t = __ldg(tw + ti0);
    w[0] = t.x;
    wsh[0] = t.y;
  } else {
    const uint4 *t4 = reinterpret_cast<const uint4 *>(tw + ti0);
#pragma unroll
    for (int g = 0; g < NG / 2; ++g) {
      const uint4 t = __ldg(t4 + g);
      w[2 * g] = t.x;
      wsh[2 * g] = t.y;
      w[2 * g + 1] = t.z;
      wsh[2 * g + 1] = t.w;
    }
  }
}

// stage LS of pass PASS (CT stage s = first_stage(PASS) + LS; the inverse runs the same
// butterfly positions with Gentleman-Sande butterflies and psi^-1 twiddles)
// SQ (small modulus, q < kSmallQ): the forward keeps every value unreduced -- a stage adds
// at most 2q to the bound, so canonical inputs stay below (2 log2(n) + 1) q < 2^32 -- and is
// reduced once after the last stage; the inverse keeps values in [0, 2q) (4q < 2^32).
template <int LOGN, int PASS, int LS, bool INV, int P_, int LE, bool SQ, int E>
__device__ __forceinline__ void ntt_stage(uint32_t (&a)[P_][E], int th, uint32_t q, const uint2 *__restrict__ tw,
                                          const InvScale &sc) {
  using P = NttPlan<LOGN, LE>;
  constexpr int rb = P::radix_bits(PASS), s0 = P::first_stage(PASS), plo = LOGN - s0 - rb;
  constexpr int s = s0 + LS, half = 1 << (rb - 1 - LS), nv = E >> rb, ng = 1 << LS;
#pragma unroll
  for (int v = 0; v < nv; ++v) {
    const int H = (v * P::T + P::template vth<PASS>(th)) >> plo;
    if constexpr (INV && s == 0) {
#pragma unroll
      for (int b = 0; b < half; ++b) {
        const int e1 = (v << rb) + b, e2 = e1 + half;
#pragma unroll
        for (int p = 0; p < P_; ++p) {
          const uint32_t U = a[p][e1], V = a[p][e2];
          a[p][e1] = shoup_mul(U + V, sc.ninv, sc.ninv_sh, q);
          a[p][e2] = shoup_mul(U - V + (SQ ? 2 * q : q), sc.w1n, sc.w1n_sh, q);
        }
      }
    } else {
      uint32_t w[ng], wsh[ng];
      load_twiddles<ng>(tw, (1 << s) + (H << LS), w, wsh);
#pragma unroll
      for (int g = 0; g < ng; ++g) {
#pragma unroll
        for (int b = 0; b < half; ++b) {
          const int e1 = (v << rb) + g * 2 * half + b, e2 = e1 + half;
#pragma unroll
          for (int p = 0; p < P_; ++p) {
            if constexpr (!INV && SQ) {
              const uint32_t V = shoup_lazy(a[p][e2], w[g], wsh[g], q);  // [0, 2q)
              const uint32_t U = a[p][e1];
              a[p][e1] = U + V;
              a[p][e2] = U - V + 2 * q;
            } else if constexpr (INV && SQ) {
              const uint32_t U = a[p][e1], V = a[p][e2];  // both in [0, 2q)
              a[p][e1] = __viaddmin_u32(U, V, U + V - 2 * q);
              a[p][e2] = shoup_lazy(U - V + 2 * q, w[g], wsh[g], q);
            } else if constexpr (!INV) {
              // An output that the next stage of this pass multiplies by a twiddle (register
              // bit half/2 set) may stay in [0, 2q): Shoup takes any input below 2^32.  The
              // others, and every output of a pass's last stage, are reduced to [0, q).  The
              // element multiplied here may arrive unreduced; U never does.
              const uint32_t V = shoup_mul(a[p][e2], w[g], wsh[g], q);
              const uint32_t U = a[p][e1];
              constexpr int nh = half >> 1;
              const bool lazy1 = (LS + 1 < rb) && ((e1 & nh) != 0);
              const bool lazy2 = (LS + 1 < rb) && ((e2 & nh) != 0);
              a[p][e1] = lazy1 ? U + V : mod_add(U, V, q);
              a[p][e2] = lazy2 ? U - V + q : mod_sub(U, V, q);
            } else {
              const uint32_t U = a[p][e1], V = a[p][e2];
              a[p][e1] = mod_add(U, V, q);
              a[p][e2] = shoup_mul(U - V + q, w[g], wsh[g], q);
            }
          }
        }
      }
    }
  }
}

template <int LOGN, int PASS, int LS, int P_, int LE, bool SQ, int E>
__device__ __forceinline__ void ntt_fwd_stages(uint32_t (&a)[P_][E], int th, uint32_t q, const uint2 *tw) {
  ntt_stage<LOGN, PASS, LS, false, P_, LE, SQ>(a, th, q, tw, InvScale{});
  if constexpr (LS + 1 < NttPlan<LOGN, LE>::radix_bits(PASS))
    ntt_fwd_stages<LOGN, PASS, LS + 1, P_, LE, SQ>(a, th, q, tw);
}
template <int LOGN, int PASS, int P_, int LE, bool SQ, int E>
__device__ __forceinline__ void ntt_fwd_passes(uint32_t (&a)[P_][E], uint32_t *sm, int th, uint32_t q,
                                               const uint2 *tw) {
  if constexpr (PASS > 0) ntt_exchange<LOGN, PASS - 1, PASS, P_, LE>(a, sm, th);
  ntt_fwd_stages<LOGN, PASS, 0, P_, LE, SQ>(a, th, q, tw);
  if constexpr (PASS + 1 < NttPlan<LOGN, LE>::NP) ntt_fwd_passes<LOGN, PASS + 1, P_, LE, SQ>(a, sm, th, q, tw);
}
template <int LOGN, int PASS, int LS, int P_, int LE, bool SQ, int E>
__device__ __forceinline__ void ntt_inv_stages(uint32_t (&a)[P_][E], int th, uint32_t q, const uint2 *tw,
                                               const InvScale &sc) {
  ntt_stage<LOGN, PASS, LS, true, P_, LE, SQ>(a, th, q, tw, sc);
  if constexpr (LS > 0) ntt_inv_stages<LOGN, PASS, LS - 1, P_, LE, SQ>(a, th, q, tw, sc);
}
template <int LOGN, int PASS, int P_, int LE, bool SQ, int E>
__device__ __forceinline__ void ntt_inv_passes(uint32_t (&a)[P_][E], uint32_t *sm, int th, uint32_t q,
                                               const uint2 *tw, const InvScale &sc) {
  if constexpr (PASS + 1 < NttPlan<LOGN, LE>::NP) ntt_exchange<LOGN, PASS + 1, PASS, P_, LE>(a, sm, th);
  ntt_inv_stages<LOGN, PASS, NttPlan<LOGN, LE>::radix_bits(PASS) - 1, P_, LE, SQ>(a, th, q, tw, sc);
  if constexpr (PASS > 0) ntt_inv_passes<LOGN, PASS - 1, P_, LE, SQ>(a, sm, th, q, tw, sc);
}

// Registers a[p][] hold the pass-0 layout on entry and the last-pass layout (E consecutive
// coefficients th*E .. th*E+E-1) on exit.  sm: P_ x SMEM_WORDS scratch for this group.
template <int LOGN, int P_, int LE = 4, bool SQ = false, int E>
__device__ __forceinline__ void ntt_fwd_core(uint32_t (&a)[P_][E], uint32_t *sm, int th, uint32_t q,
                                             const uint2 *__restrict__ psi2, uint32_t qr = 0) {
  static_assert(E == (1 << LE), "register block size");
  static_assert(!SQ || (2 * LOGN + 1) * (uint64_t)kSmallQ <= (1ull << 32), "small-modulus bound");
  ntt_fwd_passes<LOGN, 0, P_, LE, SQ>(a, sm, th, q, psi2);
  if constexpr (SQ) {  // x < (2 log2(n) + 1) q: x - floor(x qr / 2^32) q is in [0, 2q)
#pragma unroll
    for (int p = 0; p < P_; ++p)
#pragma unroll
      for (int e = 0; e < E; ++e) a[p][e] = mod_red1(a[p][e] - __umulhi(a[p][e], qr) * q, q);
  }
}
template <int LOGN>
__device__ __forceinline__ void ntt_fwd_core(uint32_t (&a)[16], uint32_t *sm, int th, uint32_t q,
                                             const uint2 *__restrict__ psi2) {
  ntt_fwd_core<LOGN, 1>(reinterpret_cast<uint32_t(&)[1][16]>(a), sm, th, q, psi2);
}

// Registers hold the last-pass layout (E consecutive coefficients) on entry and the
// pass-0 layout on exit.  Inputs must be canonical residues.
template <int LOGN, int P_, int LE = 4, bool SQ = false, int E>
__device__ __forceinline__ void ntt_inv_core(uint32_t (&a)[P_][E], uint32_t *sm, int th, uint32_t q,
                                             const uint2 *__restrict__ ipsi2, uint32_t ninv, uint32_t ninv_sh,
                                             uint32_t w1n, uint32_t w1n_sh) {
  static_assert(E == (1 << LE), "register block size");
  ntt_inv_passes<LOGN, NttPlan<LOGN, LE>::NP - 1, P_, LE, SQ>(a, sm, th, q, ipsi2,
                                                                InvScale{ninv, ninv_sh, w1n, w1n_sh});
}
template <int LOGN>
__device__ __forceinline__ void ntt_inv_core(uint32_t (&a)[16], uint32_t *sm, int th, uint32_t q,
                                             const uint2 *__restrict__ ipsi2, uint32_t ninv, uint32_t ninv_sh,
                                             uint32_t w1n, uint32_t w1n_sh) {
  ntt_inv_core<LOGN, 1>(reinterpret_cast<uint32_t(&)[1][16]>(a), sm, th, q, ipsi2, ninv, ninv_sh, w1n, w1n_sh);
}

}  // namespace cufe
