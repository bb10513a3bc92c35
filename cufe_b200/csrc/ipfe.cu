// ipfe.cu -- RNS rings, NTT launchers and the RLWE-IPFE scheme kernels (setup, encrypt,
// keygen, decrypt, decode) with their host orchestration.
//
// Scheme (reference: src/rlwe_sife.c, src/rlwe_sife_gpu.cu): ring Z_q[X]/(X^n+1), q = q0 q1 q2
// in RNS; mpk_i = a*s_i + e_i (NTT domain), c_l = INTT(a^ r^) + f_0,
// c_i = INTT(pk_i^ r^) + f_i + floor(q/p) x_i, sk_y = sum y_i s_i,
// d_y = sum y_i c_i - c_l * sk_y, decoded as round(p d_y / q).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "ctx.h"
#include "ntt.cuh"
#include "scheme.cuh"
#include "sampler_host.h"
#include "prof.h"

namespace cufe {

// ================================================================== host number theory

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = r * b % q;
    b = b * b % q;
    e >>= 1;
  }
  return r;
}
static uint64_t invmod(uint64_t a, uint64_t q) { return powmod(a, q - 2, q); }

static bool is_prime32(uint32_t n) {  // deterministic Miller-Rabin for n < 3.2e9
  if (n < 2) return false;
  for (uint32_t p : {2u, 3u, 5u, 7u})
    if (n % p == 0) return n == p;
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) d >>= 1, ++s;
  for (uint64_t a : {2ull, 3ull, 5ull, 7ull}) {
    uint64_t x = powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = x * x % n;
      if (x == n - 1) {
        comp = false;
        break;
      }
    }
    if (comp) return false;
  }
  return true;
}

static uint32_t primitive_root(uint32_t q) {
  std::vector<uint64_t> f;
  uint64_t m = q - 1;
  for (uint64_t p = 2; p * p <= m; ++p)
    if (m % p == 0) {
      f.push_back(p);
      while (m % p == 0) m /= p;
    }
  if (m > 1) f.push_back(m);
  for (uint32_t g = 2;; ++g) {
    bool ok = true;
    for (uint64_t p : f)
      if (powmod(g, (q - 1) / p, q) == 1) {
        ok = false;
        break;
      }
    if (ok) return g;
  }
}

// psi_j: primitive 8192-th roots of unity of the reference twiddle tables
// (src/consts.h: psi[j][k] = psi_j^{bitrev12(k)}, i.e. psi_j = psi[j][2048]).
static const uint32_t kPsi8192[3] = {3689u, 1689795u, 456478u};

static uint32_t root_for(uint32_t q, int n) {
  for (int j = 0; j < 3; ++j) {
    if (q != kRefPrimes[j]) continue;
    if (2 * n <= 8192) return (uint32_t)powmod(kPsi8192[j], 8192 / (2 * n), q);
    // n = 8192: the smaller square root of psi_8192 (same chain of tables)
    const uint64_t h = powmod(primitive_root(q), (q - 1) / 16384, q);
    uint64_t best = 0;
    for (uint64_t t = 1; t < 16384; t += 2) {
      const uint64_t c = powmod(h, t, q);
      if (c * c % q == kPsi8192[j] && (best == 0 || c < best)) best = c;
    }
    return (uint32_t)best;
  }
  return (uint32_t)powmod(primitive_root(q), (q - 1) / (2ull * n), q);
}

std::vector<uint32_t> ntt_primes(int k) {
  std::vector<uint32_t> v;
  for (int j = 0; j < 3 && (int)v.size() < k; ++j) v.push_back(kRefPrimes[j]);
  for (uint64_t c = ((1ull << 31) - 1) / 16384 * 16384 + 1; (int)v.size() < k; c -= 16384) {
    const uint32_t cc = (uint32_t)c;
    if (std::find(v.begin(), v.end(), cc) == v.end() && is_prime32(cc)) v.push_back(cc);
  }
  return v;
}

static unsigned bitrev(unsigned x, int bits) {
  unsigned r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

int Ring::init(int n_, int k_, const uint32_t *primes, int dev) {
  if (n_ < 16 || n_ > 8192 || (n_ & (n_ - 1)) || k_ < 1 || k_ > kMaxModuli) return CUFE_ERR_INVALID;
  n = n_;
  k = k_;
  device = dev;
  logn = 0;
  while ((1 << logn) < n) ++logn;
  q = primes ? std::vector<uint32_t>(primes, primes + k) : ntt_primes(k);
  for (uint32_t qq : q)
    if (qq >= (1u << 31) || (qq - 1) % (2u * n) != 0 || !is_prime32(qq)) return CUFE_ERR_INVALID;
  std::vector<uint32_t> tab(4 * (size_t)k * n);
  h_psi.assign((size_t)k * n, 0);
  h_ipsi.assign((size_t)k * n, 0);
  psi_root.assign(k, 0);
  std::memset(&args, 0, sizeof(args));
  std::vector<uint64_t> pw(n), ipw(n);
  for (int m = 0; m < k; ++m) {
    const uint64_t qq = q[m], w = root_for(q[m], n), wi = invmod(w, qq);
    psi_root[m] = (uint32_t)w;
    pw[0] = ipw[0] = 1;
    for (int e = 1; e < n; ++e) pw[e] = pw[e - 1] * w % qq, ipw[e] = ipw[e - 1] * wi % qq;
    for (int i = 0; i < n; ++i) {
      const uint32_t a = (uint32_t)pw[bitrev(i, logn)], b = (uint32_t)ipw[bitrev(i, logn)];
      h_psi[(size_t)m * n + i] = a;
      h_ipsi[(size_t)m * n + i] = b;
      // interleaved (w, floor(w 2^32 / q)) pairs: psi2[k][n], then ipsi2[k][n]
      tab[2 * ((size_t)m * n + i)] = a;
      tab[2 * ((size_t)m * n + i) + 1] = shoup_of(a, (uint32_t)qq);
      tab[2 * ((size_t)(k + m) * n + i)] = b;
      tab[2 * ((size_t)(k + m) * n + i) + 1] = shoup_of(b, (uint32_t)qq);
    }
    args.q[m] = (uint32_t)qq;
    args.ninv[m] = (uint32_t)invmod(n, qq);
    args.ninv_sh[m] = shoup_of(args.ninv[m], (uint32_t)qq);
    args.w1n[m] = (uint32_t)((uint64_t)h_ipsi[(size_t)m * n + 1] * args.ninv[m] % qq);
    args.w1n_sh[m] = shoup_of(args.w1n[m], (uint32_t)qq);
    args.qr[m] = (uint32_t)((1ull << 32) / qq);
  }
  args.n = n;
  args.logn = logn;
  // untuned default: the variant that measured fastest on a B200 for every n (two residues of
  // one modulus per group at 64 registers: 4 CTAs of 256 threads or 2 of 512 per SM)
  args.pp_fwd = args.pp_inv = 6;
  args.k = k;
  CUFE_CUDA(cudaSetDevice(device));
  CUFE_CUDA(cudaMalloc(&d_tab, tab.size() * 4));
  CUFE_CUDA(cudaMemcpy(d_tab, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice));
  args.psi2 = reinterpret_cast<const uint2 *>(d_tab);
  args.ipsi2 = reinterpret_cast<const uint2 *>(d_tab) + (size_t)k * n;
  return CUFE_OK;
}

void Ring::release() {
  if (d_tab) cudaFree(d_tab);
  d_tab = nullptr;
}

// ================================================================== NTT kernels

namespace {

// MODE 0 forward, 1 forward + Shoup companions into sh, 2 inverse.  data holds `rows`
// polynomials of k residues ([row][k][n]); a thread group transforms PP residues of one
// modulus m, rows PP*t .. PP*t+PP-1, sharing twiddles and shared-memory addresses.
// LBT, MINB: the launch bounds the registers are allocated for -- LBT threads per CTA (at
// least the CTA's real size) and MINB CTAs per SM.  Variant 1 uses (512, 1): at most 128
// registers; variant 2 (its CTA size, 1): up to 255, its two residues want more than 128;
// variant 4 (256, 5): 48 registers and 40 warps per SM; variants 5 and 6: two residues at
// 3 or 4 CTAs per SM (80 or 64 registers).
// the moduli one launch covers: residues r = row * k + m[i] for i < nm
struct ModSel {
  int nm;
  int m[kMaxModuli];
};

// Batched transform of rows x (selected moduli) residue polynomials, PP residues of one
// modulus per thread group.  SQ: every selected modulus is below kSmallQ (lazy butterflies);
// the launcher runs one grid over the small moduli and one over the others.
template <int LOGN, int MODE, int PP, int LBT = 512, int MINB = 1, int LE = 4, bool SQ = false>
__global__ void __launch_bounds__(LBT, MINB)
    k_ntt(uint32_t *__restrict__ data, uint32_t *__restrict__ sh, long long rows, RingArgs ra, ModSel sel) {
  using P = NttPlan<LOGN, LE>;
  constexpr int E = P::E;
  extern __shared__ uint32_t smem_u32[];
  const int th = threadIdx.x, k = ra.k, nm = sel.nm;
  const long long groups = (rows + PP - 1) / PP * nm;
  const long long gi = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const long long gg = gi < groups ? gi : groups - 1;
  const int m = sel.m[gg % nm];
  const long long row0 = gg / nm * PP;
  const uint32_t q = ra.q[m];
  uint32_t *sm = smem_u32 + threadIdx.y * PP * P::SMEM_WORDS;
  long long res[PP];
  bool live[PP];
#pragma unroll
  for (int p = 0; p < PP; ++p) {
    live[p] = gi < groups && row0 + p < rows;
    res[p] = (live[p] ? row0 + p : row0) * k + m;  // a dead slot recomputes row0, stores nothing
  }
  uint32_t a[PP][E];
  if (MODE != 2) {
#pragma unroll
    for (int p = 0; p < PP; ++p) {
      const uint32_t *d = data + res[p] * P::N;
#pragma unroll
      for (int e = 0; e < E; ++e) a[p][e] = d[P::template idx<0>(th, e)];
    }
    ntt_fwd_core<LOGN, PP, LE, SQ>(a, sm, th, q, ra.psi2 + (size_t)m * P::N, ra.qr[m]);
#pragma unroll
    for (int p = 0; p < PP; ++p) {
      if (!live[p]) continue;
      store_vec(data + res[p] * P::N + th * E, a[p]);
      if (MODE == 1) {
        uint32_t b[E];
#pragma unroll
        for (int e = 0; e < E; ++e) b[e] = (uint32_t)(((uint64_t)a[p][e] << 32) / q);
        store_vec(sh + res[p] * P::N + th * E, b);
      }
    }
  } else {
#pragma unroll
    for (int p = 0; p < PP; ++p) load_vec(data + res[p] * P::N + th * E, a[p]);
    ntt_inv_core<LOGN, PP, LE, SQ>(a, sm, th, q, ra.ipsi2 + (size_t)m * P::N, ra.ninv[m], ra.ninv_sh[m],
                                   ra.w1n[m], ra.w1n_sh[m]);
#pragma unroll
    for (int p = 0; p < PP; ++p) {
      if (!live[p]) continue;
      uint32_t *d = data + res[p] * P::N;
#pragma unroll
      for (int e = 0; e < E; ++e) d[P::template idx<0>(th, e)] = a[p][e];
    }
  }
}

template <int LOGN, int MODE, int PP, int LBT, int MINB, int LE, bool SQ>
int launch_ntt_sel(const RingArgs &ra, const ModSel &sel, uint32_t *data, uint32_t *sh, long long rows,
                   cudaStream_t s) {
  using P = NttPlan<LOGN, LE>;
  constexpr int G = ppc<LOGN, LE>();
  const size_t smem = (size_t)G * PP * P::SMEM_WORDS * 4;
  static bool attr = false;
  if (!attr) {
    CUFE_CUDA(cudaFuncSetAttribute(k_ntt<LOGN, MODE, PP, LBT, MINB, LE, SQ>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    attr = true;
  }
  const long long groups = (rows + PP - 1) / PP * sel.nm;
  const long long grid = (groups + G - 1) / G;
  if (grid <= 0) return CUFE_OK;
  note_launch(), k_ntt<LOGN, MODE, PP, LBT, MINB, LE, SQ><<<(unsigned)grid, dim3(P::T, G), smem, s>>>(data, sh, rows, ra, sel);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

// one grid over the moduli below kSmallQ (lazy butterflies), one over the rest
template <int LOGN, int MODE, int PP, int LBT = 512, int MINB = 1, int LE = 4>
int launch_ntt_pp(const RingArgs &ra, uint32_t *data, uint32_t *sh, long long rows, cudaStream_t s) {
  ModSel small{0, {}}, large{0, {}};
  for (int m = 0; m < ra.k; ++m) {
    if (ra.q[m] < kSmallQ)
      small.m[small.nm++] = m;
    else
      large.m[large.nm++] = m;
  }
  ProfScope ps(MODE == 2 ? "ntt_inverse" : "ntt_forward", s);
  int rc = CUFE_OK;
  if (small.nm) rc = launch_ntt_sel<LOGN, MODE, PP, LBT, MINB, LE, true>(ra, small, data, sh, rows, s);
  if (!rc && large.nm) rc = launch_ntt_sel<LOGN, MODE, PP, LBT, MINB, LE, false>(ra, large, data, sh, rows, s);
  return rc;
}

// Persistent form: each thread group walks residues r, r + stride, ... and issues the global
// loads of its next residue into registers before transforming the current one, so every
// CTA keeps a residue's worth of loads in flight while it computes.  One residue per thread
// group; the trip count is uniform per CTA (the exchanges synchronise the CTA).
template <int LOGN, int MODE>
__global__ void __maxnreg__(80) k_ntt_stream(uint32_t *__restrict__ data, uint32_t *__restrict__ sh,
                                                    long long nres, RingArgs ra) {
  using P = NttPlan<LOGN>;
  extern __shared__ uint32_t smem_u32[];
  const int th = threadIdx.x;
  uint32_t *sm = smem_u32 + threadIdx.y * P::SMEM_WORDS;
  const long long stride = (long long)gridDim.x * blockDim.y;
  const long long cta0 = (long long)blockIdx.x * blockDim.y;
  const long long iters = cta0 < nres ? (nres - cta0 + stride - 1) / stride : 0;
  const long long r0 = cta0 + threadIdx.y;
  uint32_t nx[16];
  {
    const uint32_t *d = data + (r0 < nres ? r0 : nres - 1) * P::N;
    if (MODE != 2) {
#pragma unroll
      for (int e = 0; e < 16; ++e) nx[e] = d[P::template idx<0>(th, e)];
    } else {
      load16(d + th * 16, nx);
    }
  }
  for (long long it = 0; it < iters; ++it) {
    const long long cur = r0 + it * stride;
    const bool act = cur < nres;
    const long long cc = act ? cur : nres - 1;
    uint32_t a[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) a[e] = nx[e];
    if (it + 1 < iters) {
      const long long nxt = cur + stride;
      const uint32_t *d = data + (nxt < nres ? nxt : nres - 1) * P::N;
      if (MODE != 2) {
#pragma unroll
        for (int e = 0; e < 16; ++e) nx[e] = d[P::template idx<0>(th, e)];
      } else {
        load16(d + th * 16, nx);
      }
    }
    const int m = (int)(cc % ra.k);
    const uint32_t q = ra.q[m];
    uint32_t *d = data + cc * P::N;
    if (MODE != 2) {
      ntt_fwd_core<LOGN>(a, sm, th, q, ra.psi2 + (size_t)m * P::N);
      if (act) {
        store16(d + th * 16, a);
        if (MODE == 1) {
          uint32_t b[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) b[e] = (uint32_t)(((uint64_t)a[e] << 32) / q);
          store16(sh + cc * P::N + th * 16, b);
        }
      }
    } else {
      ntt_inv_core<LOGN>(a, sm, th, q, ra.ipsi2 + (size_t)m * P::N, ra.ninv[m], ra.ninv_sh[m], ra.w1n[m],
                         ra.w1n_sh[m]);
      if (act) {
#pragma unroll
        for (int e = 0; e < 16; ++e) d[P::template idx<0>(th, e)] = a[e];
      }
    }
    __syncthreads();  // the next iteration's first exchange reuses sm
  }
}

inline int device_sms() {
  static int sms[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!sms[dev] && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    sms[dev] = 148;
  return sms[dev];
}

template <int LOGN, int MODE>
int launch_ntt_stream(const RingArgs &ra, uint32_t *data, uint32_t *sh, long long nres, cudaStream_t s) {
  using P = NttPlan<LOGN>;
  constexpr int G = ppc<LOGN>();
  const size_t smem = (size_t)G * P::SMEM_WORDS * 4;
  static int occ = 0;
  if (!occ) {
    CUFE_CUDA(cudaFuncSetAttribute(k_ntt_stream<LOGN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    CUFE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ntt_stream<LOGN, MODE>, P::T * G, smem));
    if (occ < 1) occ = 1;
  }
  const long long need = (nres + G - 1) / G;
  const long long grid = std::min(need, (long long)device_sms() * occ);
  if (grid <= 0) return CUFE_OK;
  ProfScope ps(MODE == 2 ? "ntt_inverse" : "ntt_forward", s);
  note_launch(), k_ntt_stream<LOGN, MODE><<<(unsigned)grid, dim3(P::T, G), smem, s>>>(data, sh, nres, ra);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

// residues per thread group: the ring's tuned choice for this direction, else 1
template <int LOGN, int MODE>
int launch_ntt_t(const RingArgs &ra, uint32_t *data, uint32_t *sh, long long nres, cudaStream_t s) {
  if (nres % ra.k) return CUFE_ERR_INVALID;
  const long long rows = nres / ra.k;
  const int pp = MODE == 2 ? ra.pp_inv : ra.pp_fwd;
  if (pp == 3) return launch_ntt_stream<LOGN, MODE>(ra, data, sh, nres, s);
  constexpr int nt = NttPlan<LOGN>::T * ppc<LOGN>();  // threads per CTA
  if (pp == 2 && rows >= 2) return launch_ntt_pp<LOGN, MODE, 2, nt, 1>(ra, data, sh, rows, s);
  if (pp == 4) return launch_ntt_pp<LOGN, MODE, 1, nt, nt <= 256 ? 5 : 2>(ra, data, sh, rows, s);
  if (pp == 5 && rows >= 2) return launch_ntt_pp<LOGN, MODE, 2, nt, nt <= 256 ? 3 : 1>(ra, data, sh, rows, s);
  if (pp == 6 && rows >= 2) return launch_ntt_pp<LOGN, MODE, 2, nt, nt <= 256 ? 4 : 2>(ra, data, sh, rows, s);
  // radix 32 and 64: 32 or 64 coefficients per thread, fewer passes and exchanges
  if constexpr (LOGN >= 10) {
    constexpr int nt5 = NttPlan<LOGN, 5>::T * ppc<LOGN, 5>();
    if (pp == 7) return launch_ntt_pp<LOGN, MODE, 1, nt5, 2, 5>(ra, data, sh, rows, s);
    if (pp == 8) return launch_ntt_pp<LOGN, MODE, 1, nt5, 3, 5>(ra, data, sh, rows, s);
  }
  if constexpr (LOGN >= 11) {
    constexpr int nt6 = NttPlan<LOGN, 6>::T * ppc<LOGN, 6>();
    if (pp == 9) return launch_ntt_pp<LOGN, MODE, 1, nt6, 2, 6>(ra, data, sh, rows, s);
  }
  return launch_ntt_pp<LOGN, MODE, 1>(ra, data, sh, rows, s);
}

template <int MODE>
int launch_ntt(const RingArgs &ra, uint32_t *data, uint32_t *sh, long long nres, cudaStream_t s) {
  switch (ra.logn) {
    case 4: return launch_ntt_t<4, MODE>(ra, data, sh, nres, s);
    case 5: return launch_ntt_t<5, MODE>(ra, data, sh, nres, s);
    case 6: return launch_ntt_t<6, MODE>(ra, data, sh, nres, s);
    case 7: return launch_ntt_t<7, MODE>(ra, data, sh, nres, s);
    case 8: return launch_ntt_t<8, MODE>(ra, data, sh, nres, s);
    case 9: return launch_ntt_t<9, MODE>(ra, data, sh, nres, s);
    case 10: return launch_ntt_t<10, MODE>(ra, data, sh, nres, s);
    case 11: return launch_ntt_t<11, MODE>(ra, data, sh, nres, s);
    case 12: return launch_ntt_t<12, MODE>(ra, data, sh, nres, s);
    case 13: return launch_ntt_t<13, MODE>(ra, data, sh, nres, s);
  }
  return CUFE_ERR_INVALID;
}

// ================================================================== scheme kernels


// mpk_i = a^ * NTT(s_i) + e^_i for residue polynomials r = 3i + m (src/rlwe_sife.c:69-76)
template <int LOGN>
__global__ void __launch_bounds__(512) k_setup_mpk(const uint32_t *__restrict__ msk, const uint32_t *__restrict__ ehat,
                                                   const uint32_t *__restrict__ ahat,
                                                   const uint32_t *__restrict__ ahat_sh, uint32_t *__restrict__ mpk,
                                                   long long nres, RingArgs ra) {
  using P = NttPlan<LOGN>;
  extern __shared__ uint32_t smem_u32[];
  const int th = threadIdx.x;
  const long long r = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const bool act = r < nres;
  const long long rr = act ? r : nres - 1;
  const int m = (int)(rr % 3);
  const uint32_t q = ra.q[m];
  uint32_t *sm = smem_u32 + threadIdx.y * P::SMEM_WORDS;
  uint32_t a[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) a[e] = msk[rr * P::N + P::template idx<0>(th, e)];
  ntt_fwd_core<LOGN>(a, sm, th, q, ra.psi2 + (size_t)m * P::N);
  uint32_t w[16], wsh[16], ev[16];
  load16(ahat + (size_t)m * P::N + th * 16, w);
  load16(ahat_sh + (size_t)m * P::N + th * 16, wsh);
  load16(ehat + rr * P::N + th * 16, ev);
#pragma unroll
  for (int e = 0; e < 16; ++e) a[e] = mod_add(shoup_mul(a[e], w[e], wsh[e], q), ev[e], q);
  if (act) store16(mpk + rr * P::N + th * 16, a);
}

// Fused encryption (src/rlwe_sife.c:157-176): for instance b and residue polynomial
// r = 3i + m of the ciphertext, c = INTT(pk_r * r^) + f + floor(q/p) x_i.  A thread group
// transforms PP instances (b, b + 1, ...) of one residue: one pk load, shared twiddles and
// exchange addresses.  Work items are residue-major so the instances of one pk polynomial run
// together (pk read once per batch).
template <int LOGN, int PP, int MINB>
__global__ void __launch_bounds__(NttPlan<LOGN>::T * ppc<LOGN>(), MINB)
    k_encrypt(const uint32_t *__restrict__ mpk, const uint32_t *__restrict__ rhat, const uint32_t *__restrict__ rhat_sh,
              long long rhat_stride, const uint32_t *__restrict__ f3, long long f3_stride,
              const uint32_t *__restrict__ f0, long long f0_stride, const uint32_t *__restrict__ x,
              uint32_t *__restrict__ ct, int batch, long long nwork, SchemeArgs sa) {
  using P = NttPlan<LOGN>;
  extern __shared__ uint32_t smem_u32[];
  const int th = threadIdx.x;
  const int bgroups = (batch + PP - 1) / PP;
  const long long wi = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const bool act = wi < nwork;
  const long long ww = act ? wi : nwork - 1;
  const int l = sa.l;
  const long long res = ww / bgroups;
  const int b0 = (int)(ww - res * bgroups) * PP;
  const int m = (int)(res % 3), i = (int)(res / 3);
  const uint32_t q = sa.ra.q[m];
  uint32_t *sm = smem_u32 + threadIdx.y * PP * P::SMEM_WORDS;
  uint32_t a[PP][16];
  {
    uint32_t pk[16];
    load16(mpk + res * P::N + th * 16, pk);
#pragma unroll
    for (int p = 0; p < PP; ++p) {
      const int b = min(b0 + p, batch - 1);  // a dead slot repeats the last instance, stores nothing
      uint32_t w[16], wsh[16];
      load16(rhat + b * rhat_stride + (size_t)m * P::N + th * 16, w);
      load16(rhat_sh + b * rhat_stride + (size_t)m * P::N + th * 16, wsh);
#pragma unroll
      for (int e = 0; e < 16; ++e) a[p][e] = shoup_mul(pk[e], w[e], wsh[e], q);
    }
  }
  ntt_inv_core<LOGN, PP>(a, sm, th, q, sa.ra.ipsi2 + (size_t)m * P::N, sa.ra.ninv[m], sa.ra.ninv_sh[m],
                         sa.ra.w1n[m], sa.ra.w1n_sh[m]);
  if (!act) return;
#pragma unroll
  for (int p = 0; p < PP; ++p) {
    const int b = b0 + p;
    if (b >= batch) break;
    const uint32_t *f;
    uint32_t msg = 0;
    if (i < l) {
      f = f3 + b * f3_stride + ((size_t)i * 3 + m) * P::N;
      const uint32_t xr = mod_u64(x[(size_t)b * l + i], sa.mu[m], q);
      msg = shoup_mul(xr, sa.delta_mod[m], sa.delta_sh[m], q);
    } else {
      f = f0 + b * f0_stride + (size_t)m * P::N;
    }
    uint32_t *c = ct + ((size_t)b * (l + 1) * 3 + res) * P::N;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int j = P::template idx<0>(th, e);
      c[j] = mod_add(mod_add(a[p][e], f[j], q), msg, q);
    }
  }
}

// sk_y = sum_i (y_i mod q_m) msk_i (src/rlwe_sife.c:215-245); KCH keys per pass over msk
template <int KCH>
__global__ void __launch_bounds__(256) k_keygen(const uint32_t *__restrict__ y, int y_signed, int nkeys,
                                                const uint32_t *__restrict__ msk, uint32_t *__restrict__ sky, int n,
                                                SchemeArgs sa) {
  extern __shared__ uint32_t smem_u32[];
  const int l = sa.l, m = blockIdx.y, k0 = blockIdx.z * KCH;
  const uint32_t q = sa.ra.q[m];
  uint32_t *yq = smem_u32, *ys = smem_u32 + KCH * l;
  for (int t = threadIdx.x; t < KCH * l; t += blockDim.x) {
    const int kk = t / l, i = t - kk * l;
    uint32_t v = 0;
    if (k0 + kk < nkeys) v = y_residue(y[(size_t)(k0 + kk) * l + i], y_signed, q, sa.mu[m]);
    yq[t] = v;
    ys[t] = (uint32_t)(((uint64_t)v << 32) / q);
  }
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint64_t acc[KCH];
#pragma unroll
  for (int kk = 0; kk < KCH; ++kk) acc[kk] = 0;
  for (int i = 0; i < l; ++i) {
    const uint32_t v = __ldg(msk + ((size_t)i * 3 + m) * n + j);
#pragma unroll
    for (int kk = 0; kk < KCH; ++kk) acc[kk] += shoup_lazy(v, yq[kk * l + i], ys[kk * l + i], q);
  }
#pragma unroll
  for (int kk = 0; kk < KCH; ++kk)
    if (k0 + kk < nkeys) sky[((size_t)(k0 + kk) * 3 + m) * n + j] = mod_u64(acc[kk], sa.mu[m], q);
}

// Decryption (src/rlwe_sife.c:248-278), d_y = sum_i y_i c_i - INTT(NTT(c_l) NTT(sk_y)), in
// two kernels.  k_dec_mac streams the ciphertexts: thread = 4 consecutive coefficients of one
// (ciphertext, key, residue), 16-byte loads, Shoup products accumulated in 64 bits; the
// l-sum is optionally split into S chunks (small batches) with canonical partial sums.
// k_dec_tail adds the chunks and subtracts the negacyclic product c_l * sk_y.
__global__ void __launch_bounds__(256) k_dec_mac(const uint32_t *__restrict__ ct, const uint32_t *__restrict__ y,
                                                 int y_signed, int nkeys, int nsplit, uint32_t *__restrict__ part,
                                                 SchemeArgs sa) {
  extern __shared__ uint32_t smem_u32[];
  const int n = sa.ra.n, l = sa.l;
  const int per_poly = n / 4 / blockDim.x;  // CTAs per residue polynomial
  const int s = blockIdx.x / per_poly, sub = blockIdx.x - s * per_poly;
  const int w = blockIdx.y;  // (c * nkeys + key) * 3 + m
  const int m = w % 3, ck = w / 3, key = ck % nkeys, c = ck / nkeys;
  const uint32_t q = sa.ra.q[m];
  const int i0 = (int)((long long)l * s / nsplit), i1 = (int)((long long)l * (s + 1) / nsplit);
  uint32_t *yq = smem_u32, *ys = smem_u32 + (i1 - i0);
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const uint32_t v = y_residue(y[(size_t)key * l + i], y_signed, q, sa.mu[m]);
    yq[i - i0] = v;
    ys[i - i0] = (uint32_t)(((uint64_t)v << 32) / q);
  }
  __syncthreads();
  const int j = 4 * (sub * blockDim.x + threadIdx.x);
  const uint32_t *cb = ct + (size_t)c * (l + 1) * 3 * n + (size_t)m * n + j;
  uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll 4
  for (int i = i0; i < i1; ++i) {
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(cb + (size_t)i * 3 * n));
    const uint32_t yv = yq[i - i0], yh = ys[i - i0];
    a0 += shoup_lazy(v.x, yv, yh, q);
    a1 += shoup_lazy(v.y, yv, yh, q);
    a2 += shoup_lazy(v.z, yv, yh, q);
    a3 += shoup_lazy(v.w, yv, yh, q);
  }
  uint4 o;
  o.x = mod_u64(a0, sa.mu[m], q);
  o.y = mod_u64(a1, sa.mu[m], q);
  o.z = mod_u64(a2, sa.mu[m], q);
  o.w = mod_u64(a3, sa.mu[m], q);
  *reinterpret_cast<uint4 *>(part + ((size_t)w * nsplit + s) * n + j) = o;
}

template <int LOGN>
__global__ void __launch_bounds__(512)
    k_dec_tail(const uint32_t *__restrict__ part, int nsplit, const uint32_t *__restrict__ clhat,
               const uint32_t *__restrict__ skhat, const uint32_t *__restrict__ skhat_sh, int nkeys,
               uint32_t *__restrict__ dy, long long nwork, SchemeArgs sa) {
  using P = NttPlan<LOGN>;
  extern __shared__ uint32_t smem_u32[];
  const int th = threadIdx.x;
  const long long wi = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const bool act = wi < nwork;
  const long long ww = act ? wi : nwork - 1;
  const int m = (int)(ww % 3);
  const long long ck = ww / 3;
  const int key = (int)(ck % nkeys), c = (int)(ck / nkeys);
  const uint32_t q = sa.ra.q[m];
  uint32_t *sm = smem_u32 + threadIdx.y * P::SMEM_WORDS;
  uint32_t a[16], w[16], wsh[16];
  load16(clhat + ((size_t)c * 3 + m) * P::N + th * 16, a);
  load16(skhat + ((size_t)key * 3 + m) * P::N + th * 16, w);
  load16(skhat_sh + ((size_t)key * 3 + m) * P::N + th * 16, wsh);
#pragma unroll
  for (int e = 0; e < 16; ++e) a[e] = shoup_mul(a[e], w[e], wsh[e], q);
  ntt_inv_core<LOGN>(a, sm, th, q, sa.ra.ipsi2 + (size_t)m * P::N, sa.ra.ninv[m],
                     sa.ra.ninv_sh[m], sa.ra.w1n[m], sa.ra.w1n_sh[m]);
  if (act) {
    const uint32_t *pp = part + (size_t)ww * nsplit * P::N;
    uint32_t *o = dy + ww * P::N;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int j = P::template idx<0>(th, e);
      uint32_t mac = pp[j];
      for (int s = 1; s < nsplit; ++s) mac = mod_add(mac, pp[(size_t)s * P::N + j], q);
      o[j] = mod_sub(mac, a[e], q);
    }
  }
}

__global__ void k_decode(const uint32_t *__restrict__ dy, int count, int ncoeff, uint32_t *__restrict__ out,
                         DecodeArgs d) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)count * ncoeff) return;
  const int cnt = (int)(gid / ncoeff), k = (int)(gid - (long long)cnt * ncoeff);
  const uint32_t *v = dy + (size_t)cnt * 3 * d.n + k;
  out[gid] = decode_one(v[0], v[d.n], v[2 * (size_t)d.n], d);
}


// Constant-coefficient decryption and decode.  The reference decodes only coefficient 0 of
// d_y (src/rlwe_sife.c:380, main.c:205 and 326), so per (ciphertext, key) and modulus
//   d_y[0] = sum_i y_i c_i[0] - (c_l * sk_y)[0],
//   (c_l * sk_y)[0] = c_l[0] sk_y[0] - sum_{t=1}^{n-1} c_l[t] sk_y[n-t]   (negacyclic),
// equal to coefficient 0 of the full decryption (src/rlwe_sife.c:248-286) residue for residue.
// One CTA per (ciphertext, key); reads l + 2n words per modulus instead of (l+1) n.
__global__ void __launch_bounds__(256)
    k_dec_coef0(const uint32_t *__restrict__ ct, const uint32_t *__restrict__ y, int y_signed, int nkeys,
                const uint32_t *__restrict__ sky, uint32_t *__restrict__ d0, uint32_t *__restrict__ out,
                SchemeArgs sa, DecodeArgs dd) {
  __shared__ uint64_t red[8];
  const int n = sa.ra.n, l = sa.l;
  const int key = blockIdx.x % nkeys, c = blockIdx.x / nkeys;
  const uint32_t *cb = ct + (size_t)c * (l + 1) * 3 * n;
  uint32_t r[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const uint32_t q = sa.ra.q[m];
    const uint64_t mu = sa.mu[m];
    uint64_t mac = 0, neg = 0;
    for (int i = threadIdx.x; i < l; i += blockDim.x) {
      const uint32_t yv = y_residue(y[(size_t)key * l + i], y_signed, q, mu);
      mac += mod_u64((uint64_t)cb[((size_t)i * 3 + m) * n] * yv, mu, q);
    }
    const uint32_t *cl = cb + ((size_t)l * 3 + m) * n;
    const uint32_t *sk = sky + ((size_t)key * 3 + m) * n;
    for (int t = threadIdx.x + 1; t < n; t += blockDim.x) neg += mod_u64((uint64_t)cl[t] * sk[n - t], mu, q);
    const uint64_t macs = block_sum_u64(mac, red), negs = block_sum_u64(neg, red);
    const uint32_t c0s0 = mod_u64((uint64_t)cl[0] * sk[0], mu, q);
    // mac - (c_l[0] s[0] - neg)
    r[m] = mod_add(mod_sub(mod_u64(macs, mu, q), c0s0, q), mod_u64(negs, mu, q), q);
  }
  if (threadIdx.x == 0) {
    if (d0) {
      d0[(size_t)blockIdx.x * 3 + 0] = r[0];
      d0[(size_t)blockIdx.x * 3 + 1] = r[1];
      d0[(size_t)blockIdx.x * 3 + 2] = r[2];
    }
    out[blockIdx.x] = decode_one(r[0], r[1], r[2], dd);
  }
}

// Constant-coefficient decrypt of many (ciphertext, key) pairs as a tiled product over K =
// l + n: for modulus m = blockIdx.z,
//   d0[c][key][m] = sum_{k<l} c_k[0] y_k + sum_{t<n} c_l[t] b_t,  b_0 = -s[0], b_t = s[n-t],
// the negacyclic constant term of c_l * sk_y with its sign folded into the key operand.  A CTA of
// 256 threads computes TM = 16 RI ciphertexts x TN = 16 RJ keys, RI x RJ per thread, from
// 32-deep K chunks staged in shared memory (A reused TN times, B TM times); the rows are
// XOR-swizzled in steps of the vector width so that the staging stores spread over the banks.
// Products are exact: a, b < 2^31, so four products sum below 2^64 in one wide multiply-add
// chain, folded into a 64 + 32-bit accumulator (K < 2^34 products); one reduction per pair.
// Tile shapes (ciphertexts x keys): 64 x 32 (the default), 64 x 64, 32 x 32, 32 x 64; the
// context's tuner picks per (ciphertexts, keys).
constexpr int kC0Kc = 32;
constexpr int kCoef0TiledMinKeys = 32;  // fewer keys: one CTA per pair (untuned rule)
constexpr int kCoef0Forms = 5;          // 0 per pair, 1..4 the tile shapes below
template <int TM, int R>
__device__ __forceinline__ int c0_swz(int kk, int i) {
  return kk * TM + (i ^ ((kk & (TM / R - 1)) * R));
}
template <int R>
__device__ __forceinline__ void c0_row(const uint32_t *p, uint32_t (&v)[R]) {
  if constexpr (R == 4) {
    const uint4 t = *reinterpret_cast<const uint4 *>(p);
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else {
    const uint2 t = *reinterpret_cast<const uint2 *>(p);
    v[0] = t.x, v[1] = t.y;
  }
}

template <int RI, int RJ>
__global__ void __launch_bounds__(256) k_dec_coef0_tiled(const uint32_t *__restrict__ ct, const uint32_t *__restrict__ y,
                                                         int y_signed, int nct, int nkeys,
                                                         const uint32_t *__restrict__ sky, uint32_t *__restrict__ d0,
                                                         SchemeArgs sa) {
  constexpr int TM = 16 * RI, TN = 16 * RJ;
  __shared__ __align__(16) uint32_t As[kC0Kc * TM];
  __shared__ __align__(16) uint32_t Bs[kC0Kc * TN];
  const int m = blockIdx.z, n = sa.ra.n, l = sa.l, K = l + n;
  const uint32_t q = sa.ra.q[m];
  const uint64_t mu = sa.mu[m];
  const int ct0 = blockIdx.x * TM, key0 = blockIdx.y * TN;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  uint64_t lo[RI][RJ];
  uint32_t hi[RI][RJ];
#pragma unroll
  for (int i = 0; i < RI; ++i)
#pragma unroll
    for (int j = 0; j < RJ; ++j) lo[i][j] = 0, hi[i][j] = 0;
  for (int k0 = 0; k0 < K; k0 += kC0Kc) {
    // lane-consecutive k: the c_l and sk_y parts are contiguous runs per row
    for (int e = threadIdx.x; e < TM * kC0Kc; e += blockDim.x) {
      const int i = e / kC0Kc, kk = e % kC0Kc, k = k0 + kk, c = ct0 + i;
      uint32_t a = 0;
      if (k < K && c < nct) {
        const uint32_t *cb = ct + (size_t)c * (l + 1) * 3 * n;
        a = k < l ? cb[((size_t)k * 3 + m) * n] : cb[((size_t)l * 3 + m) * n + (k - l)];
      }
      As[c0_swz<TM, RI>(kk, i)] = a;
    }
    for (int e = threadIdx.x; e < TN * kC0Kc; e += blockDim.x) {
      const int j = e / kC0Kc, kk = e % kC0Kc, k = k0 + kk, key = key0 + j;
      uint32_t b = 0;
      if (k < K && key < nkeys) {
        if (k < l) {
          b = y_residue(y[(size_t)key * l + k], y_signed, q, mu);
        } else {
          const uint32_t *sk = sky + ((size_t)key * 3 + m) * n;
          const int t = k - l;
          b = t == 0 ? (sk[0] ? q - sk[0] : 0u) : sk[n - t];
        }
      }
      Bs[c0_swz<TN, RJ>(kk, j)] = b;
    }
    __syncthreads();
#pragma unroll 2
    for (int kk = 0; kk < kC0Kc; kk += 4) {
      uint32_t a[4][RI], b[4][RJ];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        c0_row<RI>(&As[c0_swz<TM, RI>(kk + u, ty * RI)], a[u]);
        c0_row<RJ>(&Bs[c0_swz<TN, RJ>(kk + u, tx * RJ)], b[u]);
      }
#pragma unroll
      for (int i = 0; i < RI; ++i)
#pragma unroll
        for (int j = 0; j < RJ; ++j) {
          uint64_t t = (uint64_t)a[0][i] * b[0][j];
#pragma unroll
          for (int u = 1; u < 4; ++u) t += (uint64_t)a[u][i] * b[u][j];
          const uint64_t nl = lo[i][j] + t;
          hi[i][j] += nl < t;
          lo[i][j] = nl;
        }
    }
    __syncthreads();
  }
  const uint64_t c64 = 0ull - mu * q;  // 2^64 mod q
#pragma unroll
  for (int i = 0; i < RI; ++i) {
    const int c = ct0 + ty * RI + i;
#pragma unroll
    for (int j = 0; j < RJ; ++j) {
      const int key = key0 + tx * RJ + j;
      if (c < nct && key < nkeys)
        d0[((size_t)c * nkeys + key) * 3 + m] = mod_u64(mod_u64(lo[i][j], mu, q) + (uint64_t)hi[i][j] * c64, mu, q);
    }
  }
}

// decode of coefficient-0 residue triples d0[p][3] -> out[p]
__global__ void k_decode_triples(const uint32_t *__restrict__ d0, long long npairs, uint32_t *__restrict__ out,
                                 DecodeArgs dd) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npairs) out[p] = decode_one(d0[p * 3], d0[p * 3 + 1], d0[p * 3 + 2], dd);
}

}  // namespace

int ntt_launch(const RingArgs &ra, uint32_t *data, long long nres, bool inverse, cudaStream_t s) {
  return inverse ? launch_ntt<2>(ra, data, nullptr, nres, s) : launch_ntt<0>(ra, data, nullptr, nres, s);
}
int ntt_fwd_shoup_launch(const RingArgs &ra, uint32_t *data, uint32_t *sh, long long nres, cudaStream_t s) {
  return launch_ntt<1>(ra, data, sh, nres, s);
}

int ring_tune(Ring &r, long long npoly, float *ms, cudaStream_t s) {
  const size_t poly_bytes = (size_t)r.k * r.n * 4;
  npoly = std::max(2LL, std::min(npoly, (long long)((1ull << 30) / poly_bytes)));
  uint32_t *buf = nullptr;
  CUFE_CUDA(cudaMalloc(&buf, (size_t)npoly * poly_bytes));
  // zero residues: the kernels' instruction stream does not depend on the values
  cudaError_t err = cudaMemsetAsync(buf, 0, (size_t)npoly * poly_bytes, s);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  constexpr int NV = CUFE_NTT_VARIANTS;
  float t[2 * NV] = {};
  int rc = CUFE_OK;
  if (err == cudaSuccess) err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  const RingArgs saved = r.args;
  for (int i = 0; i < 2 * NV && err == cudaSuccess && rc == CUFE_OK; ++i) {
    const bool inv = i >= NV;
    r.args.pp_fwd = r.args.pp_inv = 1 + i % NV;
    const long long nres = npoly * r.k;
    rc = ntt_launch(r.args, buf, nres, inv, s);  // warm-up
    if (rc) break;
    if ((err = cudaEventRecord(e0, s)) != cudaSuccess) break;
    for (int rep = 0; rep < 3 && rc == CUFE_OK; ++rep) rc = ntt_launch(r.args, buf, nres, inv, s);
    if (rc || (err = cudaEventRecord(e1, s)) != cudaSuccess || (err = cudaEventSynchronize(e1)) != cudaSuccess) break;
    if ((err = cudaEventElapsedTime(&t[i], e0, e1)) != cudaSuccess) break;
    t[i] /= 3.0f;
  }
  r.args = saved;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  if (rc) return rc;
  if (err != cudaSuccess) {
    set_last_error(std::string("ring_tune: ") + cudaGetErrorString(err));
    return CUFE_ERR_CUDA;
  }
  int bf = 0, bi = NV;
  for (int v = 1; v < NV; ++v) {
    if (t[v] < t[bf]) bf = v;
    if (t[NV + v] < t[bi]) bi = NV + v;
  }
  r.args.pp_fwd = 1 + bf;
  r.args.pp_inv = 1 + bi - NV;
  if (ms)
    for (int i = 0; i < 2 * NV; ++i) ms[i] = t[i];
  return CUFE_OK;
}

// ================================================================== context

int Ctx::init(int n_, int l_, int dev) {
  if (l_ < 1 || l_ > 65536) return CUFE_ERR_INVALID;
  n = n_;
  l = l_;
  device = dev;
  int rc = ring.init(n_, 3, kRefPrimes, dev);
  if (rc) return rc;
  CUFE_CUDA(cudaSetDevice(device));
  CUFE_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  CUFE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CUFE_CUDA(cudaMalloc(&d_status, 256));
  CUFE_CUDA(cudaMemset(d_status, 0, 256));
  rc = sampler_init_device();
  if (rc) return rc;
  p = 4u * 16u * (uint32_t)l + 1u;  // B_x * B_y * l + 1 (src/params.h:26)
  q = (u128)kRefPrimes[0] * kRefPrimes[1] * kRefPrimes[2];
  qhalf = q / 2;
  const u128 delta = q / p;  // floor(q/p) (src/params.h:27)
  for (int j = 0; j < 3; ++j) {
    delta_mod[j] = (uint32_t)(delta % kRefPrimes[j]);
    delta_sh[j] = shoup_of(delta_mod[j], kRefPrimes[j]);
  }
  crt_c1 = (uint32_t)invmod(kRefPrimes[0], kRefPrimes[1]);
  crt_c2 = (uint32_t)invmod((uint64_t)kRefPrimes[0] * kRefPrimes[1] % kRefPrimes[2], kRefPrimes[2]);
  crt_c1_sh = shoup_of(crt_c1, kRefPrimes[1]);
  crt_c2_sh = shoup_of(crt_c2, kRefPrimes[2]);
  return CUFE_OK;
}

void Ctx::release() {
  if (ws) cudaFree(ws);
  if (d_status) cudaFree(d_status);
  if (stream) cudaStreamDestroy(stream);
  ring.release();
  ws = nullptr;
  d_status = nullptr;
  stream = nullptr;
}

int Ctx::ensure_ws(size_t bytes) {
  if (bytes <= ws_bytes) return CUFE_OK;
  CUFE_CUDA(cudaDeviceSynchronize());
  if (ws) CUFE_CUDA(cudaFree(ws));
  ws = nullptr;
  ws_bytes = 0;
  const size_t want = bytes + (bytes >> 3);
  if (cudaMalloc(&ws, want) != cudaSuccess) {
    cudaGetLastError();
    set_last_error("workspace allocation of " + std::to_string(want) + " bytes failed");
    return CUFE_ERR_NOMEM;
  }
  ws_bytes = want;
  return CUFE_OK;
}

int Ctx::check_status(cudaStream_t s) {
  uint32_t st = 0;
  CUFE_CUDA(cudaMemcpyAsync(&st, d_status, 4, cudaMemcpyDeviceToHost, s));
  CUFE_CUDA(cudaStreamSynchronize(s));
  if (st) {
    CUFE_CUDA(cudaMemsetAsync(d_status, 0, 4, s));
    std::string why;
    if (st & 1u) why += " uniform draw beyond the refill buffer;";
    if (st & 2u) why += " precomputed refill range exhausted;";
    if (st & 4u) why += " GPU-mapping refill cap reached;";
    if (st & 8u) why += " candidate at or above 2^33;";
    set_last_error(std::string("sampler status ") + std::to_string(st) + ":" + why);
    return CUFE_ERR_SAMPLER;
  }
  return CUFE_OK;
}

static SchemeArgs scheme_args(const Ctx &c) {
  SchemeArgs sa;
  sa.ra = c.ring.args;
  sa.l = c.l;
  for (int j = 0; j < 3; ++j) {
    sa.delta_mod[j] = c.delta_mod[j];
    sa.delta_sh[j] = c.delta_sh[j];
    sa.mu[j] = (uint64_t)(((u128)1 << 64) / kRefPrimes[j]);
  }
  return sa;
}

struct Arena {
  uint8_t *p;
  size_t used = 0;
  explicit Arena(uint8_t *base) : p(base) {}
  template <class T>
  T *take(size_t count) {
    T *r = reinterpret_cast<T *>(p + used);
    used += (count * sizeof(T) + 255) & ~(size_t)255;
    return r;
  }
};

static std::vector<uint32_t> expand_keys(int count, const uint8_t *keys) {
  std::vector<uint32_t> rk((size_t)count * 60, 0u);  // null keys: all-zero schedule
  if (keys)
    for (int i = 0; i < count; ++i) aes_key_expand(keys + 32 * (size_t)i, rk.data() + 60 * (size_t)i);
  return rk;
}

template <class F>
static int dispatch_logn(int logn, F &&f) {
  switch (logn) {
    case 4: return f(std::integral_constant<int, 4>());
    case 5: return f(std::integral_constant<int, 5>());
    case 6: return f(std::integral_constant<int, 6>());
    case 7: return f(std::integral_constant<int, 7>());
    case 8: return f(std::integral_constant<int, 8>());
    case 9: return f(std::integral_constant<int, 9>());
    case 10: return f(std::integral_constant<int, 10>());
    case 11: return f(std::integral_constant<int, 11>());
    case 12: return f(std::integral_constant<int, 12>());
    case 13: return f(std::integral_constant<int, 13>());
  }
  return CUFE_ERR_INVALID;
}

// shared tail of both setups: a^ = NTT(a) in place, e^ = NTT(e), mpk_i = a^ NTT(s_i) + e^_i
static int setup_tail(Ctx &c, int l, uint32_t *d_mpk, const uint32_t *d_msk, uint32_t *e, uint32_t *a_sh,
                      cudaStream_t s) {
  const int n = c.n;
  uint32_t *ahat = d_mpk + (size_t)l * 3 * n;
  int rc = ntt_fwd_shoup_launch(c.ring.args, ahat, a_sh, 3, s);
  if (rc) return rc;
  rc = ntt_launch(c.ring.args, e, (long long)l * 3, false, s);
  if (rc) return rc;
  const long long nres = (long long)l * 3;
  return dispatch_logn(c.ring.logn, [&](auto L) {
    constexpr int LOGN = decltype(L)::value;
    constexpr int G = ppc<LOGN>();
    CUFE_CUDA(cudaFuncSetAttribute(k_setup_mpk<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    ProfScope ps("setup_mpk", s);
    note_launch(), k_setup_mpk<LOGN><<<(unsigned)((nres + G - 1) / G), dim3(NttPlan<LOGN>::T, G), G * NttPlan<LOGN>::SMEM_WORDS * 4, s>>>(
        d_msk, e, ahat, a_sh, d_mpk, nres, c.ring.args);
    CUFE_CUDA(cudaGetLastError());
    return CUFE_OK;
  });
}

int ctx_setup_cpu_map(Ctx &c, const uint8_t *seed_a, const uint8_t *seed_s, const uint8_t *seed_e, uint32_t *d_mpk,
                      uint32_t *d_msk, cudaStream_t s) {
  return ctx_setup_cpu_map_l(c, c.l, seed_a, seed_s, seed_e, d_mpk, d_msk, s);
}

int ctx_setup_cpu_map_l(Ctx &c, int l, const uint8_t *seed_a, const uint8_t *seed_s, const uint8_t *seed_e,
                        uint32_t *d_mpk, uint32_t *d_msk, cudaStream_t s) {
  if (l < 1 || !seed_a || !seed_e) return CUFE_ERR_INVALID;
  const int n = c.n;
  const size_t poly = (size_t)3 * n;
  const size_t samp_ws = cpu_map_workspace_bytes(2, l, n, 0);
  int rc = c.ensure_ws(samp_ws + (2 * l + 2) * poly * 4 + 4096 + 4 * 60 * 4);
  if (rc) return rc;
  Arena ar(c.ws);
  uint32_t *rk = ar.take<uint32_t>(3 * 60);
  uint32_t *se = ar.take<uint32_t>(2 * (size_t)l * poly);  // [2][l][3][n]: s, e
  uint32_t *a_sh = ar.take<uint32_t>(poly);
  void *sws = ar.take<uint8_t>(samp_ws);
  std::vector<uint32_t> keys(3 * 60, 0u);
  aes_key_expand(seed_a, keys.data());
  if (seed_s) aes_key_expand(seed_s, keys.data() + 60);
  aes_key_expand(seed_e, keys.data() + 120);
  CUFE_CUDA(cudaMemcpyAsync(rk, keys.data(), keys.size() * 4, cudaMemcpyHostToDevice, s));
  rc = sample_polya(rk, n, d_mpk + (size_t)l * poly, s);
  if (rc) return rc;
  rc = sample_cpu_map(0, 2, rk + 60, l, n, se, sws, c.d_status, c.num_sms, s);
  if (rc) return rc;
  CUFE_CUDA(cudaMemcpyAsync(d_msk, se, (size_t)l * poly * 4, cudaMemcpyDeviceToDevice, s));
  return setup_tail(c, l, d_mpk, d_msk, se + (size_t)l * poly, a_sh, s);
}

int ctx_setup_gpu_map(Ctx &c, const uint8_t *seed2, const uint8_t *seed3, uint32_t *d_mpk, uint32_t *d_msk,
                      cudaStream_t s) {
  const int n = c.n, l = c.l;
  const size_t poly = (size_t)3 * n;
  int rc = c.ensure_ws((size_t)(l + 1) * poly * 4 + 4096 + 2 * 60 * 4);
  if (rc) return rc;
  Arena ar(c.ws);
  uint32_t *rk = ar.take<uint32_t>(2 * 60);
  uint32_t *e = ar.take<uint32_t>((size_t)l * poly);
  uint32_t *a_sh = ar.take<uint32_t>(poly);
  std::vector<uint32_t> keys(2 * 60, 0u);
  aes_key_expand(seed2, keys.data());
  aes_key_expand(seed3, keys.data() + 60);
  CUFE_CUDA(cudaMemcpyAsync(rk, keys.data(), keys.size() * 4, cudaMemcpyHostToDevice, s));
  rc = sample_gpu_map(0, rk, 0, l, n, d_msk, c.d_status, s);
  if (rc) return rc;
  rc = sample_gpu_map(0, rk + 60, 0, l, n, e, c.d_status, s);
  if (rc) return rc;
  return setup_tail(c, l, d_mpk, d_msk, e, a_sh, s);
}

static int encrypt_tail(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint32_t *rhat,
                        const uint32_t *rhat_sh, long long rhat_stride, const uint32_t *f3, long long f3_stride,
                        const uint32_t *f0, long long f0_stride, uint32_t *d_ct, cudaStream_t s) {
  const long long nwork = (long long)(c.l + 1) * 3 * batch;
  const SchemeArgs sa = scheme_args(c);
  return dispatch_logn(c.ring.logn, [&](auto L) {
    constexpr int LOGN = decltype(L)::value;
    constexpr int G = ppc<LOGN>(), NT = NttPlan<LOGN>::T * G;
    constexpr int MINB = NT >= 1024 ? 1 : 1024 / NT;  // 64 registers
    ProfScope ps("encrypt_intt", s);
    // instances per thread group: the tuner's choice for this batch size, else two from batch 2
    int group = batch >= 2 ? 2 : 1;
    if (c.enc_group_forced) {
      group = c.enc_group_forced;
    } else {
      const auto it = c.enc_group.find(batch);
      if (it != c.enc_group.end()) group = it->second;
    }
    if (group == 2 && batch >= 2) {  // two instances per thread group
      auto kern = k_encrypt<LOGN, 2, MINB>;
      const long long nw = (long long)(c.l + 1) * 3 * ((batch + 1) / 2);
      CUFE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
      note_launch(), kern<<<(unsigned)((nw + G - 1) / G), dim3(NttPlan<LOGN>::T, G), G * 2 * NttPlan<LOGN>::SMEM_WORDS * 4, s>>>(
          d_mpk, rhat, rhat_sh, rhat_stride, f3, f3_stride, f0, f0_stride, d_x, d_ct, batch, nw, sa);
    } else {
      auto kern = k_encrypt<LOGN, 1, MINB>;
      CUFE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
      note_launch(), kern<<<(unsigned)((nwork + G - 1) / G), dim3(NttPlan<LOGN>::T, G), G * NttPlan<LOGN>::SMEM_WORDS * 4, s>>>(
          d_mpk, rhat, rhat_sh, rhat_stride, f3, f3_stride, f0, f0_stride, d_x, d_ct, batch, nwork, sa);
    }
    CUFE_CUDA(cudaGetLastError());
    return CUFE_OK;
  });
}

size_t encrypt_workspace_bytes(int n, int l, int batch) {
  const size_t poly = (size_t)3 * n;
  return cpu_map_workspace_bytes(batch, l, n, 2) + cpu_map_workspace_bytes(batch, 2, n, 1) +
         (size_t)batch * ((size_t)l * poly + 2 * poly + 2 * poly) * 4 + (size_t)batch * 2 * 60 * 4 + 16 * 256;
}

int ctx_encrypt_cpu_map(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                        const uint8_t *seeds3, uint32_t *d_ct, cudaStream_t s) {
  if (batch < 1 || !seeds2) return CUFE_ERR_INVALID;
  const int n = c.n, l = c.l;
  const size_t poly = (size_t)3 * n;
  const size_t ws3 = cpu_map_workspace_bytes(batch, l, n, 2), ws2 = cpu_map_workspace_bytes(batch, 2, n, 1);
  int rc = c.ensure_ws(encrypt_workspace_bytes(n, l, batch));
  if (rc) return rc;
  Arena ar(c.ws);
  uint32_t *rk = ar.take<uint32_t>((size_t)batch * 2 * 60);
  uint32_t *f3 = ar.take<uint32_t>((size_t)batch * l * poly);
  uint32_t *s2o = ar.take<uint32_t>((size_t)batch * 2 * poly);  // [b][2][3][n]: r, f0
  uint32_t *rhat = ar.take<uint32_t>((size_t)batch * poly);
  uint32_t *rhat_sh = ar.take<uint32_t>((size_t)batch * poly);
  void *sws3 = ar.take<uint8_t>(ws3);
  void *sws2 = ar.take<uint8_t>(ws2);
  std::vector<uint32_t> k2 = expand_keys(batch, seeds2), k3 = expand_keys(batch, seeds3);
  k2.insert(k2.end(), k3.begin(), k3.end());
  CUFE_CUDA(cudaMemcpyAsync(rk, k2.data(), k2.size() * 4, cudaMemcpyHostToDevice, s));
  rc = sample_cpu_map(1, batch, rk, 2, n, s2o, sws2, c.d_status, c.num_sms, s);
  if (rc) return rc;
  rc = sample_cpu_map(2, batch, rk + (size_t)batch * 60, l, n, f3, sws3, c.d_status, c.num_sms, s);
  if (rc) return rc;
  CUFE_CUDA(cudaMemcpy2DAsync(rhat, poly * 4, s2o, 2 * poly * 4, poly * 4, batch, cudaMemcpyDeviceToDevice, s));
  rc = ntt_fwd_shoup_launch(c.ring.args, rhat, rhat_sh, (long long)batch * 3, s);
  if (rc) return rc;
  return encrypt_tail(c, batch, d_x, d_mpk, rhat, rhat_sh, (long long)poly, f3, (long long)l * poly, s2o + poly,
                      (long long)2 * poly, d_ct, s);
}

int ctx_encrypt_gpu_map(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seed2,
                        uint32_t *d_ct, cudaStream_t s) {
  if (batch < 1 || !seed2) return CUFE_ERR_INVALID;
  const int n = c.n, l = c.l;
  const size_t poly = (size_t)3 * n;
  int rc = c.ensure_ws(((size_t)l * poly + 3 * poly) * 4 + 60 * 4 + 8 * 256);
  if (rc) return rc;
  Arena ar(c.ws);
  uint32_t *rk = ar.take<uint32_t>(60);
  uint32_t *f3 = ar.take<uint32_t>((size_t)l * poly);
  uint32_t *r = ar.take<uint32_t>(poly);
  uint32_t *rhat = ar.take<uint32_t>(poly);
  uint32_t *rhat_sh = ar.take<uint32_t>(poly);
  uint32_t keys[60];
  aes_key_expand(seed2, keys);
  CUFE_CUDA(cudaMemcpyAsync(rk, keys, sizeof(keys), cudaMemcpyHostToDevice, s));
  // r and f_0 come from the same key and counters (src/rlwe_sife_gpu.cu:135-147), f_i from the
  // same key with polynomial index i (src/sample_gpu.cu:217-289); every instance shares them.
  rc = sample_gpu_map(1, rk, 0, 1, n, r, c.d_status, s);
  if (rc) return rc;
  rc = sample_gpu_map(2, rk, 0, l, n, f3, c.d_status, s);
  if (rc) return rc;
  CUFE_CUDA(cudaMemcpyAsync(rhat, r, poly * 4, cudaMemcpyDeviceToDevice, s));
  rc = ntt_fwd_shoup_launch(c.ring.args, rhat, rhat_sh, 3, s);
  if (rc) return rc;
  return encrypt_tail(c, batch, d_x, d_mpk, rhat, rhat_sh, 0, f3, 0, r, 0, d_ct, s);
}

int ctx_keygen(Ctx &c, int nkeys, const uint32_t *d_y, int y_signed, const uint32_t *d_msk, uint32_t *d_sky,
               cudaStream_t s) {
  if (nkeys < 1) return CUFE_ERR_INVALID;
  constexpr int KCH = 4;
  const SchemeArgs sa = scheme_args(c);
  const size_t smem = (size_t)2 * KCH * c.l * 4;
  if (smem > 200 * 1024) return CUFE_ERR_INVALID;
  CUFE_CUDA(cudaFuncSetAttribute(k_keygen<KCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((c.n + 255) / 256, 3, (nkeys + KCH - 1) / KCH);
  ProfScope ps("keygen", s);
  note_launch(), k_keygen<KCH><<<grid, 256, smem, s>>>(d_y, y_signed, nkeys, d_msk, d_sky, c.n, sa);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

int ctx_decrypt(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                const uint32_t *d_sky, uint32_t *d_dy, cudaStream_t s) {
  if (nct < 1 || nkeys < 1) return CUFE_ERR_INVALID;
  const int n = c.n, l = c.l;
  const size_t poly = (size_t)3 * n;
  const long long nwork = (long long)nct * nkeys * 3;
  // split the l-sum until about two waves of MAC threads are resident
  const long long base_threads = nwork * (n / 4);
  const long long want = (long long)c.num_sms * 2048 * 2;
  int nsplit = 1;
  while (nsplit < 32 && base_threads * nsplit < want && l / (nsplit * 2) >= 8) nsplit *= 2;
  int rc = c.ensure_ws(((size_t)nct * poly + 2 * (size_t)nkeys * poly + (size_t)nwork * nsplit * n) * 4 + 8 * 256);
  if (rc) return rc;
  Arena ar(c.ws);
  uint32_t *clhat = ar.take<uint32_t>((size_t)nct * poly);
  uint32_t *skhat = ar.take<uint32_t>((size_t)nkeys * poly);
  uint32_t *skhat_sh = ar.take<uint32_t>((size_t)nkeys * poly);
  uint32_t *part = ar.take<uint32_t>((size_t)nwork * nsplit * n);
  CUFE_CUDA(cudaMemcpy2DAsync(clhat, poly * 4, d_ct + (size_t)l * poly, (size_t)(l + 1) * poly * 4, poly * 4, nct,
                              cudaMemcpyDeviceToDevice, s));
  rc = ntt_launch(c.ring.args, clhat, (long long)nct * 3, false, s);
  if (rc) return rc;
  CUFE_CUDA(cudaMemcpyAsync(skhat, d_sky, (size_t)nkeys * poly * 4, cudaMemcpyDeviceToDevice, s));
  rc = ntt_fwd_shoup_launch(c.ring.args, skhat, skhat_sh, (long long)nkeys * 3, s);
  if (rc) return rc;
  const SchemeArgs sa = scheme_args(c);
  {
    const int threads = std::min(256, n / 4);
    const int per_poly = n / 4 / threads;
    const size_t smem = (size_t)2 * ((l + nsplit - 1) / nsplit + 1) * 4;
    if (smem > 200 * 1024) return CUFE_ERR_INVALID;
    CUFE_CUDA(cudaFuncSetAttribute(k_dec_mac, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ProfScope ps("decrypt_mac", s);
    note_launch(), k_dec_mac<<<dim3(per_poly * nsplit, (unsigned)nwork), threads, smem, s>>>(d_ct, d_y, y_signed, nkeys, nsplit,
                                                                             part, sa);
    CUFE_CUDA(cudaGetLastError());
  }
  return dispatch_logn(c.ring.logn, [&](auto L) {
    constexpr int LOGN = decltype(L)::value;
    constexpr int G = ppc<LOGN>();
    const size_t smem = (size_t)G * NttPlan<LOGN>::SMEM_WORDS * 4;
    CUFE_CUDA(cudaFuncSetAttribute(k_dec_tail<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    ProfScope ps("decrypt_tail", s);
    note_launch(), k_dec_tail<LOGN><<<(unsigned)((nwork + G - 1) / G), dim3(NttPlan<LOGN>::T, G), smem, s>>>(
        part, nsplit, clhat, skhat, skhat_sh, nkeys, d_dy, nwork, sa);
    CUFE_CUDA(cudaGetLastError());
    return (int)CUFE_OK;
  });
}

// ------------------------------------------------------------------ decryption without allocation
//
// Some callers cannot call cudaMalloc while they decrypt: a host application that hands this
// library a fixed GPU memory budget up front, or a latency-critical serving thread that must
// not take the implicit device synchronisation of a cudaMalloc/cudaFree.  For them,
// ctx_decrypt_noalloc runs the same decryption kernels as ctx_decrypt with every scratch
// buffer carved from the file-scope array below instead of the context workspace.  The
// array is a fixed part of the library image: every GPU that loads the library holds its
// 2 MiB until the process exits.
constexpr int kNoAllocMaxN = 4096;    // ring degree
constexpr int kNoAllocMaxKeys = 4;    // keys per call (one ciphertext per call)
constexpr int kNoAllocMaxSplit = 8;   // chunks of the l-sum
constexpr size_t kNoAllocWords = (size_t)3 * kNoAllocMaxN                       // NTT(c_l)
                                 + (size_t)2 * kNoAllocMaxKeys * 3 * kNoAllocMaxN  // NTT(sk_y), Shoup
                                 + (size_t)3 * kNoAllocMaxKeys * kNoAllocMaxSplit * kNoAllocMaxN  // partials
                                 + 4 * 64;                                          // region padding
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// Host code may not use g_noalloc_scratch as an address: it is only a host-side stand-in for
// the symbol.  The device address comes from cudaGetSymbolAddress, once per device, with that
// device current (the first call on a device does it; make that first call before any stream
// capture).
static std::mutex g_noalloc_mu;
static uint32_t *g_noalloc_dev[64] = {};

static int noalloc_scratch(int device, uint32_t **out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= 64) return CUFE_ERR_INVALID;
  if (!g_noalloc_dev[device]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_last_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
      return CUFE_ERR_CUDA;
    }
    g_noalloc_dev[device] = static_cast<uint32_t *>(ptr);
  }
  *out = g_noalloc_dev[device];
  return CUFE_OK;
}

int ctx_decrypt_noalloc(Ctx &c, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                        const uint32_t *d_sky, uint32_t *d_dy, cudaStream_t s) {
  const int n = c.n, l = c.l;
  if (n > kNoAllocMaxN || nkeys < 1 || nkeys > kNoAllocMaxKeys) {
    set_last_error("cufe_decrypt_noalloc supports n <= " + std::to_string(kNoAllocMaxN) + " and 1.." +
                   std::to_string(kNoAllocMaxKeys) + " keys per call (got n = " + std::to_string(n) +
                   ", keys = " + std::to_string(nkeys) + ")");
    return CUFE_ERR_INVALID;
  }
  uint32_t *base = nullptr;
  int rc = noalloc_scratch(c.device, &base);
  if (rc) return rc;
  const size_t poly = (size_t)3 * n;
  const long long nwork = (long long)nkeys * 3;
  const long long base_threads = nwork * (n / 4);
  const long long want = (long long)c.num_sms * 2048 * 2;
  int nsplit = 1;
  while (nsplit < kNoAllocMaxSplit && base_threads * nsplit < want && l / (nsplit * 2) >= 8) nsplit *= 2;
  auto round64 = [](size_t w) { return (w + 63) & ~(size_t)63; };
  uint32_t *clhat = base;
  uint32_t *skhat = clhat + round64(poly);
  uint32_t *skhat_sh = skhat + round64((size_t)nkeys * poly);
  uint32_t *part = skhat_sh + round64((size_t)nkeys * poly);
  // every scratch word read below is written first by this call (no zeroing needed)
  CUFE_CUDA(cudaMemcpyAsync(clhat, d_ct + (size_t)l * poly, poly * 4, cudaMemcpyDeviceToDevice, s));
  rc = ntt_launch(c.ring.args, clhat, 3, false, s);
  if (rc) return rc;
  CUFE_CUDA(cudaMemcpyAsync(skhat, d_sky, (size_t)nkeys * poly * 4, cudaMemcpyDeviceToDevice, s));
  rc = ntt_fwd_shoup_launch(c.ring.args, skhat, skhat_sh, (long long)nkeys * 3, s);
  if (rc) return rc;
  const SchemeArgs sa = scheme_args(c);
  {
    const int threads = std::min(256, n / 4);
    const int per_poly = n / 4 / threads;
    const size_t smem = (size_t)2 * ((l + nsplit - 1) / nsplit + 1) * 4;
    if (smem > 200 * 1024) return CUFE_ERR_INVALID;
    CUFE_CUDA(cudaFuncSetAttribute(k_dec_mac, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    note_launch(), k_dec_mac<<<dim3(per_poly * nsplit, (unsigned)nwork), threads, smem, s>>>(d_ct, d_y, y_signed, nkeys, nsplit,
                                                                             part, sa);
    CUFE_CUDA(cudaGetLastError());
  }
  return dispatch_logn(c.ring.logn, [&](auto L) {
    constexpr int LOGN = decltype(L)::value;
    constexpr int G = ppc<LOGN>();
    const size_t smem = (size_t)G * NttPlan<LOGN>::SMEM_WORDS * 4;
    CUFE_CUDA(cudaFuncSetAttribute(k_dec_tail<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    note_launch(), k_dec_tail<LOGN><<<(unsigned)((nwork + G - 1) / G), dim3(NttPlan<LOGN>::T, G), smem, s>>>(
        part, nsplit, clhat, skhat, skhat_sh, nkeys, d_dy, nwork, sa);
    CUFE_CUDA(cudaGetLastError());
    return (int)CUFE_OK;
  });
}

static DecodeArgs decode_args(const Ctx &c) {
  DecodeArgs d;
  d.q0 = kRefPrimes[0];
  d.q1 = kRefPrimes[1];
  d.q2 = kRefPrimes[2];
  d.c1 = c.crt_c1;
  d.c1_sh = c.crt_c1_sh;
  d.c2 = c.crt_c2;
  d.c2_sh = c.crt_c2_sh;
  d.mu2 = (uint64_t)(((u128)1 << 64) / kRefPrimes[2]);
  d.q01 = (uint64_t)kRefPrimes[0] * kRefPrimes[1];
  d.qlo = (unsigned long long)(uint64_t)c.q;
  d.qhi = (unsigned long long)(uint64_t)(c.q >> 64);
  d.hlo = (unsigned long long)(uint64_t)c.qhalf;
  d.hhi = (unsigned long long)(uint64_t)(c.qhalf >> 64);
  d.p = c.p;
  d.n = c.n;
  return d;
}

int ctx_decode(Ctx &c, int count, const uint32_t *d_dy, int ncoeff, uint32_t *d_out, cudaStream_t s) {
  if (count < 1 || ncoeff < 1 || ncoeff > c.n) return CUFE_ERR_INVALID;
  const DecodeArgs d = decode_args(c);
  const long long total = (long long)count * ncoeff;
  ProfScope ps("decode", s);
  note_launch(), k_decode<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(d_dy, count, ncoeff, d_out, d);
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

// the tiled product with RI x RJ pairs per thread
template <int RI, int RJ>
static int launch_coef0_tiled(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                              const uint32_t *d_sky, uint32_t *d0, cudaStream_t s) {
  const dim3 grid((unsigned)((nct + 16 * RI - 1) / (16 * RI)), (unsigned)((nkeys + 16 * RJ - 1) / (16 * RJ)), 3);
  note_launch(), k_dec_coef0_tiled<RI, RJ><<<grid, 256, 0, s>>>(d_ct, d_y, y_signed, nct, nkeys, d_sky, d0,
                                                                  scheme_args(c));
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

// form 0: one CTA per (ciphertext, key) pair; 1..4: the tiled product at 64x32, 64x64, 32x32,
// 32x64 (ciphertexts x keys) then the decode of every pair
int ctx_decrypt_coef0_form(Ctx &c, int form, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y,
                           int y_signed, const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, cudaStream_t s) {
  if (nct < 1 || nkeys < 1 || (long long)nct * nkeys > 0x7fffffffLL || !d_out || form < 0 || form >= kCoef0Forms)
    return CUFE_ERR_INVALID;
  if (form == 0) {
    ProfScope ps("decrypt_coef0", s);
    note_launch(), k_dec_coef0<<<(unsigned)(nct * nkeys), 256, 0, s>>>(d_ct, d_y, y_signed, nkeys, d_sky, d_d0, d_out,
                                                        scheme_args(c), decode_args(c));
    CUFE_CUDA(cudaGetLastError());
    return CUFE_OK;
  }
  // many keys per ciphertext: the tiled product, then the decode of every pair
  const long long npairs = (long long)nct * nkeys;
  uint32_t *d0 = d_d0;
  if (!d0) {
    const int rc = c.ensure_ws((size_t)npairs * 3 * 4);
    if (rc) return rc;
    d0 = reinterpret_cast<uint32_t *>(c.ws);
  }
  ProfScope ps("decrypt_coef0", s);
  int rc = CUFE_OK;
  if (form == 1) rc = launch_coef0_tiled<4, 2>(c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d0, s);
  if (form == 2) rc = launch_coef0_tiled<4, 4>(c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d0, s);
  if (form == 3) rc = launch_coef0_tiled<2, 2>(c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d0, s);
  if (form == 4) rc = launch_coef0_tiled<2, 4>(c, nct, d_ct, nkeys, d_y, y_signed, d_sky, d0, s);
  if (rc) return rc;
  note_launch(), k_decode_triples<<<(unsigned)((npairs + 255) / 256), 256, 0, s>>>(d0, npairs, d_out, decode_args(c));
  CUFE_CUDA(cudaGetLastError());
  return CUFE_OK;
}

// device time of one call of f() on s after one untimed call (the better of two timed calls)
template <class F>
static int time_call(F f, cudaStream_t s, float *ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CUFE_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    set_last_error("tuner: cudaEventCreate failed");
    return CUFE_ERR_CUDA;
  }
  int rc = f();
  float best = 0;
  for (int rep = 0; rep < 2 && rc == CUFE_OK; ++rep) {
    float t = 0;
    if (cudaEventRecord(e0, s) != cudaSuccess || (rc = f()) != CUFE_OK) break;
    if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
      set_last_error("tuner: event timing failed");
      rc = CUFE_ERR_CUDA;
      break;
    }
    best = rep == 0 ? t : std::min(best, t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

int ctx_tune_encrypt(Ctx &c, int batch, const uint32_t *d_x, const uint32_t *d_mpk, const uint8_t *seeds2,
                     const uint8_t *seeds3, uint32_t *d_ct, int *choice, float *ms, cudaStream_t s) {
  if (batch < 1 || !seeds2) return CUFE_ERR_INVALID;
  float t[2] = {0, 0};
  int rc = CUFE_OK;
  for (int g = 1; g <= 2 && rc == CUFE_OK; ++g) {
    c.enc_group_forced = g;
    rc = time_call([&] { return ctx_encrypt_cpu_map(c, batch, d_x, d_mpk, seeds2, seeds3, d_ct, s); }, s, &t[g - 1]);
  }
  c.enc_group_forced = 0;
  if (rc) return rc;
  const int best = (batch >= 2 && t[1] < t[0]) ? 2 : 1;
  c.enc_group[batch] = best;
  if (choice) *choice = best;
  if (ms) ms[0] = t[0], ms[1] = t[1];
  return CUFE_OK;
}

int ctx_tune_decrypt_coef0(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                           const uint32_t *d_sky, uint32_t *d_out, int *choice, float *ms, cudaStream_t s) {
  if (nct < 1 || nkeys < 1 || !d_out) return CUFE_ERR_INVALID;
  float t[kCoef0Forms] = {};
  int best = 0;
  for (int f = 0; f < kCoef0Forms; ++f) {
    const int rc = time_call(
        [&] { return ctx_decrypt_coef0_form(c, f, nct, d_ct, nkeys, d_y, y_signed, d_sky, nullptr, d_out, s); }, s,
        &t[f]);
    if (rc) return rc;
    if (t[f] < t[best]) best = f;
  }
  c.coef0_form[{nct, nkeys}] = best;
  if (choice) *choice = best;
  if (ms)
    for (int f = 0; f < kCoef0Forms; ++f) ms[f] = t[f];
  return CUFE_OK;
}

int ctx_decrypt_coef0(Ctx &c, int nct, const uint32_t *d_ct, int nkeys, const uint32_t *d_y, int y_signed,
                      const uint32_t *d_sky, uint32_t *d_d0, uint32_t *d_out, cudaStream_t s) {
  const auto it = c.coef0_form.find({nct, nkeys});
  const int form = it != c.coef0_form.end() ? it->second : (nkeys < kCoef0TiledMinKeys ? 0 : 1);
  return ctx_decrypt_coef0_form(c, form, nct, d_ct, nkeys, d_y, y_signed, d_sky, d_d0, d_out, s);
}

int ctx_sample_cpu_map(Ctx &c, int sig, int nstreams, const uint8_t *keys, int calls, uint32_t *d_out,
                       cudaStream_t s) {
  if (sig < 0 || sig > 2 || nstreams < 1 || calls < 1) return CUFE_ERR_INVALID;
  const size_t sws = cpu_map_workspace_bytes(nstreams, calls, c.n, sig);
  int rc = c.ensure_ws(sws + (size_t)nstreams * 60 * 4 + 512);
  if (rc) return rc;
  Arena ar(c.ws);
  uint32_t *rk = ar.take<uint32_t>((size_t)nstreams * 60);
  void *w = ar.take<uint8_t>(sws);
  std::vector<uint32_t> k = expand_keys(nstreams, keys);
  CUFE_CUDA(cudaMemcpyAsync(rk, k.data(), k.size() * 4, cudaMemcpyHostToDevice, s));
  return sample_cpu_map(sig, nstreams, rk, calls, c.n, d_out, w, c.d_status, c.num_sms, s);
}

int ctx_sample_gpu_map(Ctx &c, int sig, const uint8_t *key, int poly0, int npolys, uint32_t *d_out,
                       cudaStream_t s) {
  if (sig < 0 || sig > 2 || npolys < 1 || poly0 < 0 || !key) return CUFE_ERR_INVALID;
  int rc = c.ensure_ws(256 + 60 * 4);
  if (rc) return rc;
  uint32_t k[60];
  aes_key_expand(key, k);
  CUFE_CUDA(cudaMemcpyAsync(c.ws, k, sizeof(k), cudaMemcpyHostToDevice, s));
  return sample_gpu_map(sig, reinterpret_cast<uint32_t *>(c.ws), poly0, npolys, c.n, d_out, c.d_status, s);
}

int ctx_sample_polya(Ctx &c, const uint8_t *seed, uint32_t *d_a, cudaStream_t s) {
  if (!seed) return CUFE_ERR_INVALID;
  int rc = c.ensure_ws(256 + 60 * 4);
  if (rc) return rc;
  uint32_t k[60];
  aes_key_expand(seed, k);
  CUFE_CUDA(cudaMemcpyAsync(c.ws, k, sizeof(k), cudaMemcpyHostToDevice, s));
  return sample_polya(reinterpret_cast<uint32_t *>(c.ws), c.n, d_a, s);
}

}  // namespace cufe
