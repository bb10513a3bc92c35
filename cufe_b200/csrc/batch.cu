// batch.cu -- heterogeneous batches of IPFE instances.
//
// A batch holds `count` independent instances of the scheme (src/rlwe_sife.c:32-286), each
// with its own ring degree n_i, vector length l_i (so its own p_i = 64 l_i + 1 and
// Delta_i = floor(q / p_i), src/params.h:26-27) and its own master key pair, resident on the
// device.  One step runs, for every instance, encrypt(x_i) with the CPU stream mapping
// (per-instance seeds), keygen(y_i), decryption and decode of coefficient 0 -- the
// inner product -- as a fixed sequence of launches over all instances at once:
//
//   keys:     device AES-256 key expansion of every instance's two seeds
//   keygen:   one launch over (instance, modulus, 256 coefficients) units
//   per chunk of instances (scratch bounded by max_chunk_bytes):
//     sigma_2 sampler over all chunk streams (segmented CPU mapping: 2 calls of n_i each)
//     r^ = NTT(r) per ring degree
//     sigma_3 sampler over all chunk streams (l_i calls of n_i each)
//     encryption: one launch per ring degree over every (instance, slot, modulus) residue
//     constant-coefficient decryption + decode, one CTA per instance
//
// Instances are kept in ring-degree order internally (stable); inputs and outputs use the
// caller's order.  Every table the launches read is built once at creation, so a step is
// free of host work and can be captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "ctx.h"
#include "ntt.cuh"
#include "prof.h"
#include "sampler_host.h"
#include "scheme.cuh"

namespace cufe {

struct InstDev {
  uint64_t mpk, msk, sky;    // word offsets: key arena, function-key arena
  uint64_t ct, f3, s2o, rh;  // word offsets in the chunk arenas
  uint64_t x;                // word offset of x_i and y_i in the packed inputs
  uint32_t l, n, user, p;
  uint32_t delta_mod[3], delta_sh[3];
};

struct ModQ {
  uint32_t q[3];
  uint64_t mu[3];
};

namespace {

// sk_i[m][c] = sum_{j < l_i} (y_ij mod q_m) msk_i[j][m][c] (src/rlwe_sife.c:215-245); one CTA
// per (instance, modulus, 256 coefficients)
__global__ void __launch_bounds__(256)
    k_keygen_het(const InstDev *__restrict__ inst, const uint64_t *__restrict__ unit_off, uint32_t count,
                 const uint32_t *__restrict__ keys, const int32_t *__restrict__ y, uint32_t *__restrict__ sky,
                 ModQ mq) {
  extern __shared__ uint32_t smem_u32[];
  const uint32_t i = seg_find(unit_off, count, blockIdx.x);
  const InstDev I = inst[i];
  const uint32_t local = blockIdx.x - (uint32_t)unit_off[i], chunks = I.n / 256;
  const int m = (int)(local / chunks);
  const uint32_t col = (local - m * chunks) * 256 + threadIdx.x;
  const uint32_t q = mq.q[m];
  uint32_t *yq = smem_u32, *ys = smem_u32 + I.l;
  for (uint32_t j = threadIdx.x; j < I.l; j += blockDim.x) {
    const uint32_t v = y_residue((uint32_t)y[I.x + j], 1, q, mq.mu[m]);
    yq[j] = v;
    ys[j] = (uint32_t)(((uint64_t)v << 32) / q);
  }
  __syncthreads();
  const uint32_t *mk = keys + I.msk + (size_t)m * I.n + col;
  const size_t stride = (size_t)3 * I.n;
  // eight slots' loads issued ahead of their products, two partial sums: enough bytes in
  // flight per SM to keep HBM busy (one load per slot in a plain loop reached 46% of it)
  uint64_t acc0 = 0, acc1 = 0;
  uint32_t j = 0;
  for (; j + 8 <= I.l; j += 8) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = __ldg(mk + (size_t)(j + u) * stride);
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
      acc0 += shoup_lazy(v[u], yq[j + u], ys[j + u], q);
      acc1 += shoup_lazy(v[u + 1], yq[j + u + 1], ys[j + u + 1], q);
    }
  }
  for (; j < I.l; ++j) acc0 += shoup_lazy(__ldg(mk + (size_t)j * stride), yq[j], ys[j], q);
  sky[I.sky + (size_t)m * I.n + col] = mod_u64(acc0 + acc1, mq.mu[m], q);  // < 4096 * 2q < 2^44
}

// encryption of every residue (instance, slot j <= l_i, modulus m) of one ring degree
// (src/rlwe_sife.c:157-176): c = INTT(pk_j r^) + f + Delta_i x_ij, with f = f_j (sigma_3) for
// j < l_i and f_0 (the second sigma_2 call) for the last slot
template <int LOGN>
__global__ void __launch_bounds__(512)
    k_encrypt_het(const InstDev *__restrict__ inst, const uint64_t *__restrict__ res_off, uint32_t cnt,
                  long long nres, const uint32_t *__restrict__ keys, const uint32_t *__restrict__ rh,
                  const uint32_t *__restrict__ rh_sh, const uint32_t *__restrict__ f3,
                  const uint32_t *__restrict__ s2o, const uint32_t *__restrict__ x, uint32_t *__restrict__ ct,
                  RingArgs ra, ModQ mq) {
  using P = NttPlan<LOGN>;
  extern __shared__ uint32_t smem_u32[];
  const int th = threadIdx.x;
  const long long wi = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const bool act = wi < nres;
  const long long ww = act ? wi : nres - 1;
  const uint32_t i = seg_find(res_off, cnt, (uint64_t)ww);
  const InstDev &I = inst[i];
  const uint32_t local = (uint32_t)(ww - (long long)res_off[i]);
  const uint32_t j = local / 3, l = I.l;
  const int m = (int)(local - j * 3);
  const uint32_t q = ra.q[m];
  uint32_t *sm = smem_u32 + threadIdx.y * P::SMEM_WORDS;
  uint32_t a[16], w[16], wsh[16];
  load16(keys + I.mpk + (size_t)local * P::N + th * 16, a);
  load16(rh + I.rh + (size_t)m * P::N + th * 16, w);
  load16(rh_sh + I.rh + (size_t)m * P::N + th * 16, wsh);
#pragma unroll
  for (int e = 0; e < 16; ++e) a[e] = shoup_mul(a[e], w[e], wsh[e], q);
  ntt_inv_core<LOGN>(a, sm, th, q, ra.ipsi2 + (size_t)m * P::N, ra.ninv[m], ra.ninv_sh[m], ra.w1n[m],
                     ra.w1n_sh[m]);
  const uint32_t *f;
  uint32_t msg = 0;
  if (j < l) {
    f = f3 + I.f3 + (size_t)local * P::N;
    const uint32_t xr = mod_u64(x[I.x + j], mq.mu[m], q);
    msg = shoup_mul(xr, I.delta_mod[m], I.delta_sh[m], q);
  } else {
    f = s2o + I.s2o + (size_t)(3 + m) * P::N;
  }
  uint32_t *c = ct + I.ct + (size_t)local * P::N;
  if (act) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int jj = P::template idx<0>(th, e);
      c[jj] = mod_add(mod_add(a[e], f[jj], q), msg, q);
    }
  }
}

// d_y[0] = sum_j y_j c_j[0] - (c_l[0] sk[0] - sum_{t>=1} c_l[t] sk[n-t]) per modulus, then the
// reference's decode with this instance's p (src/rlwe_sife.c:248-332): one CTA per instance
__global__ void __launch_bounds__(256)
    k_dec_coef0_het(const InstDev *__restrict__ inst, const uint32_t *__restrict__ ct,
                    const uint32_t *__restrict__ sky, const int32_t *__restrict__ y, uint32_t *__restrict__ out,
                    uint32_t *__restrict__ d0, ModQ mq, DecodeArgs dd) {
  __shared__ uint64_t red[8];
  const InstDev I = inst[blockIdx.x];
  const uint32_t n = I.n, l = I.l;
  const uint32_t *cb = ct + I.ct;
  uint32_t r[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const uint32_t q = mq.q[m];
    const uint64_t mu = mq.mu[m];
    uint64_t mac = 0, neg = 0;
    for (uint32_t j = threadIdx.x; j < l; j += blockDim.x) {
      const uint32_t yv = y_residue((uint32_t)y[I.x + j], 1, q, mu);
      mac += mod_u64((uint64_t)cb[((size_t)j * 3 + m) * n] * yv, mu, q);
    }
    const uint32_t *cl = cb + ((size_t)l * 3 + m) * n;
    const uint32_t *sk = sky + I.sky + (size_t)m * n;
    for (uint32_t t = threadIdx.x + 1; t < n; t += blockDim.x) neg += mod_u64((uint64_t)cl[t] * sk[n - t], mu, q);
    const uint64_t macs = block_sum_u64(mac, red), negs = block_sum_u64(neg, red);
    const uint32_t c0s0 = mod_u64((uint64_t)cl[0] * sk[0], mu, q);
    r[m] = mod_add(mod_sub(mod_u64(macs, mu, q), c0s0, q), mod_u64(negs, mu, q), q);
  }
  if (threadIdx.x == 0) {
    if (d0)
      for (int m = 0; m < 3; ++m) d0[(size_t)I.user * 3 + m] = r[m];
    DecodeArgs d = dd;
    d.p = I.p;
    d.n = (int)n;
    out[I.user] = decode_one(r[0], r[1], r[2], d);
  }
}

template <class F>
int dispatch_logn_b(int logn, F &&f) {
  switch (logn) {
    case 8: return f(std::integral_constant<int, 8>());
    case 9: return f(std::integral_constant<int, 9>());
    case 10: return f(std::integral_constant<int, 10>());
    case 11: return f(std::integral_constant<int, 11>());
    case 12: return f(std::integral_constant<int, 12>());
    case 13: return f(std::integral_constant<int, 13>());
  }
  return CUFE_ERR_INVALID;
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// ---------------------------------------------------------------------------- host side

struct BatchGroup {  // instances of one ring degree inside a chunk
  int logn = 0;
  uint32_t first = 0, count = 0;  // chunk-local instance range
  uint64_t rh = 0, s2o = 0;       // word offsets of the group in the chunk arenas
  long long nres = 0;             // residues to encrypt: sum (l_i + 1) * 3
  size_t inst_off = 0, res_off = 0;  // byte offsets of its tables in the table blob
};

struct BatchChunk {
  uint32_t first = 0, count = 0;  // internal-order instance range
  std::vector<BatchGroup> groups;
  size_t inst_off = 0;            // byte offset of the chunk's InstDev[count]
  size_t seg2_off = 0, seg3_off = 0;
  SegSizes z2{}, z3{};
};

struct Batch {
  int device = 0, count = 0, num_sms = 148;
  std::vector<int> n, l;         // caller order
  std::vector<uint32_t> order;   // internal position -> caller index
  std::vector<int> pos_of;       // caller index -> internal position
  bool keys_only = false;        // hold keys only (no step scratch): the request server's tenants
  std::vector<uint64_t> x_off;   // caller order, count + 1
  std::map<int, std::unique_ptr<Ctx>> ctx;  // one context (ring, setup workspace) per n
  std::vector<BatchChunk> chunks;
  std::vector<InstDev> inst;     // internal order, arena offsets of the first chunk layout
  size_t scratch_bytes = 0, key_bytes = 0;
  // device memory
  uint32_t *keys = nullptr, *sky = nullptr;
  uint8_t *tables = nullptr;     // InstDev arrays, offsets, segment tables
  uint8_t *scratch = nullptr;    // chunk arenas + sampler scratch
  uint32_t *rk = nullptr;        // [2][count][60] round keys (internal order)
  uint32_t *perm = nullptr;      // internal position -> caller index
  uint32_t *status = nullptr;
  size_t keygen_inst_off = 0, keygen_unit_off = 0;
  uint32_t keygen_units = 0, max_l = 0;
  // chunk arena layout (bytes)
  size_t a_s2o = 0, a_rh = 0, a_rhsh = 0, a_f3 = 0, a_ct = 0, a_samp = 0;
  // bound inputs / outputs
  const uint32_t *x = nullptr;
  const int32_t *y = nullptr;
  const uint8_t *seeds2 = nullptr, *seeds3 = nullptr;
  uint32_t *out = nullptr, *d0 = nullptr;
  bool ran = false;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int last_chunk = -1;
  ModQ mq{};
  DecodeArgs dd{};

  size_t chunk_budget = 0;       // scratch budget the chunks were laid out for
  uint64_t sky_words = 0;
  int create(int count_, const int *n_, const int *l_, size_t max_chunk_bytes, int dev);
  int layout(size_t max_chunk_bytes);
  int tune(int nb, const size_t *budgets, size_t *chosen, float *ms, cudaStream_t s);
  void release();
  int setup(const uint8_t *sa, const uint8_t *ss, const uint8_t *se, cudaStream_t s);
  int run(cudaStream_t s);
  int replay(cudaStream_t s);
  void drop_graph();
};

static uint32_t delta_of(uint32_t p, int j) {
  const u128 q = (u128)kRefPrimes[0] * kRefPrimes[1] * kRefPrimes[2];
  return (uint32_t)((q / p) % kRefPrimes[j]);
}

int Batch::create(int count_, const int *n_, const int *l_, size_t max_chunk_bytes, int dev) {
  if (count_ < 1 || !n_ || !l_) return CUFE_ERR_INVALID;
  count = count_;
  device = dev;
  n.assign(n_, n_ + count);
  l.assign(l_, l_ + count);
  for (int i = 0; i < count; ++i) {
    if (n[i] < 256 || n[i] > 8192 || (n[i] & (n[i] - 1)) || l[i] < 1 || l[i] > 4096) {
      set_last_error("batch: n must be a power of two in [256, 8192] and l in [1, 4096]");
      return CUFE_ERR_INVALID;
    }
  }
  CUFE_CUDA(cudaSetDevice(device));
  CUFE_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  if (!max_chunk_bytes) max_chunk_bytes = (size_t)24 << 30;
  // contexts per ring degree
  for (int i = 0; i < count; ++i)
    if (!ctx.count(n[i])) {
      std::unique_ptr<Ctx> c(new Ctx);
      int rc = c->init(n[i], l[i], device);
      if (rc) return rc;
      ctx[n[i]] = std::move(c);
    }
  const Ctx &c0 = *ctx.begin()->second;
  for (int j = 0; j < 3; ++j) {
    mq.q[j] = kRefPrimes[j];
    mq.mu[j] = (uint64_t)(((u128)1 << 64) / kRefPrimes[j]);
  }
  dd.q0 = kRefPrimes[0];
  dd.q1 = kRefPrimes[1];
  dd.q2 = kRefPrimes[2];
  dd.c1 = c0.crt_c1;
  dd.c1_sh = c0.crt_c1_sh;
  dd.c2 = c0.crt_c2;
  dd.c2_sh = c0.crt_c2_sh;
  dd.mu2 = mq.mu[2];
  dd.q01 = (uint64_t)kRefPrimes[0] * kRefPrimes[1];
  dd.qlo = (unsigned long long)(uint64_t)c0.q;
  dd.qhi = (unsigned long long)(uint64_t)(c0.q >> 64);
  dd.hlo = (unsigned long long)(uint64_t)c0.qhalf;
  dd.hhi = (unsigned long long)(uint64_t)(c0.qhalf >> 64);
  // caller-order packing of x / y
  x_off.assign(count + 1, 0);
  for (int i = 0; i < count; ++i) x_off[i + 1] = x_off[i] + l[i];
  // internal order: by ring degree, stable
  order.resize(count);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return n[a] < n[b]; });
  pos_of.assign(count, 0);
  for (int pos = 0; pos < count; ++pos) pos_of[order[pos]] = pos;
  // key arena: mpk_i [(l+1)][3][n], msk_i [l][3][n]; function keys [3][n]
  inst.assign(count, InstDev{});
  uint64_t kw = 0, skw = 0;
  for (int pos = 0; pos < count; ++pos) {
    const uint32_t u = order[pos];
    InstDev &I = inst[pos];
    I.l = (uint32_t)l[u];
    I.n = (uint32_t)n[u];
    I.user = u;
    I.p = 64u * I.l + 1u;  // B_x * B_y * l + 1 with B_x = 4, B_y = 16 (src/params.h:26)
    for (int j = 0; j < 3; ++j) {
      I.delta_mod[j] = delta_of(I.p, j);
      I.delta_sh[j] = shoup_of(I.delta_mod[j], kRefPrimes[j]);
    }
    I.mpk = kw;
    kw += (uint64_t)(I.l + 1) * 3 * I.n;
    I.msk = kw;
    kw += (uint64_t)I.l * 3 * I.n;
    I.sky = skw;
    skw += (uint64_t)3 * I.n;
    I.x = x_off[u];
    max_l = std::max(max_l, I.l);
  }
  key_bytes = kw * 4;
  sky_words = skw;
  int rc = layout(max_chunk_bytes);
  if (rc) return rc;
  CUFE_CUDA(cudaMalloc(&keys, std::max<size_t>(key_bytes, 256)));
  CUFE_CUDA(cudaMalloc(&sky, std::max<size_t>(sky_words * 4, 256)));
  CUFE_CUDA(cudaMalloc(&rk, (size_t)2 * count * 60 * 4));
  CUFE_CUDA(cudaMalloc(&perm, (size_t)count * 4));
  CUFE_CUDA(cudaMemcpy(perm, order.data(), (size_t)count * 4, cudaMemcpyHostToDevice));
  CUFE_CUDA(cudaMalloc(&status, 256));
  CUFE_CUDA(cudaMemset(status, 0, 256));
  return CUFE_OK;
}

// Chunks (greedy in internal order under the scratch budget), their tables and the step
// scratch; keys and bound buffers are untouched, so a batch can be re-chunked at any time.
int Batch::layout(size_t max_chunk_bytes) {
  drop_graph();
  if (tables) cudaFree(tables);
  if (scratch) cudaFree(scratch);
  tables = scratch = nullptr;
  chunks.clear();
  chunk_budget = max_chunk_bytes;
  auto inst_bytes = [&](const InstDev &I) {
    const uint64_t poly = (uint64_t)3 * I.n * 4;
    const uint64_t R3 = cpu_map_refills(I.l, I.n, 2), R2 = cpu_map_refills(2, I.n, 1);
    return poly * (2 + 2 + I.l + (I.l + 1)) + R3 * 70 + R2 * 70 + 4096;
  };
  for (int pos = 0; pos < count;) {
    BatchChunk ch;
    ch.first = pos;
    uint64_t b = 0;
    while (pos < count && (ch.count == 0 || b + inst_bytes(inst[pos]) <= max_chunk_bytes)) {
      b += inst_bytes(inst[pos]);
      ++pos;
      ++ch.count;
    }
    chunks.push_back(ch);
  }
  // per chunk: arena offsets, groups, segment tables; sizes of the largest chunk
  std::vector<uint8_t> blob;
  auto put = [&](const void *src, size_t bytes) {
    const size_t off = a256(blob.size());
    blob.resize(off + a256(bytes));
    if (src) std::memcpy(blob.data() + off, src, bytes);
    return off;
  };
  size_t m_s2o = 0, m_rh = 0, m_f3 = 0, m_ct = 0, m_samp = 0;
  std::vector<InstDev> chunk_inst;
  for (BatchChunk &ch : chunks) {
    uint64_t w_s2o = 0, w_rh = 0, w_f3 = 0, w_ct = 0;
    std::vector<uint32_t> calls2, n2, calls3, n3;
    std::vector<uint64_t> o2, o3;
    chunk_inst.assign(inst.begin() + ch.first, inst.begin() + ch.first + ch.count);
    for (uint32_t k = 0; k < ch.count; ++k) {
      InstDev &I = chunk_inst[k];
      const int logn = __builtin_ctz(I.n);
      if (ch.groups.empty() || ch.groups.back().logn != logn) {
        BatchGroup g;
        g.logn = logn;
        g.first = k;
        g.rh = w_rh;
        g.s2o = w_s2o;
        ch.groups.push_back(g);
      }
      BatchGroup &g = ch.groups.back();
      ++g.count;
      g.nres += (long long)(I.l + 1) * 3;
      I.s2o = w_s2o;
      I.rh = w_rh;
      I.f3 = w_f3;
      I.ct = w_ct;
      calls2.push_back(2);
      n2.push_back(I.n);
      o2.push_back(w_s2o);
      calls3.push_back(I.l);
      n3.push_back(I.n);
      o3.push_back(w_f3);
      w_s2o += (uint64_t)6 * I.n;
      w_rh += (uint64_t)3 * I.n;
      w_f3 += (uint64_t)I.l * 3 * I.n;
      w_ct += (uint64_t)(I.l + 1) * 3 * I.n;
    }
    // the host copy keeps the first chunk's arena offsets (ciphertext lookup of a one-chunk batch)
    if (&ch == &chunks.front())
      for (uint32_t k = 0; k < ch.count; ++k) inst[ch.first + k] = chunk_inst[k];
    ch.inst_off = put(chunk_inst.data(), chunk_inst.size() * sizeof(InstDev));
    for (BatchGroup &g : ch.groups) {
      g.inst_off = put(chunk_inst.data() + g.first, (size_t)g.count * sizeof(InstDev));
      std::vector<uint64_t> ro(g.count + 1, 0);
      for (uint32_t k = 0; k < g.count; ++k) ro[k + 1] = ro[k] + (uint64_t)(chunk_inst[g.first + k].l + 1) * 3;
      g.res_off = put(ro.data(), ro.size() * 8);
    }
    const SegLayout L2 = seg_layout(ch.count), L3 = seg_layout(ch.count);
    std::vector<uint8_t> t2(L2.bytes), t3(L3.bytes);
    ch.z2 = seg_fill_host(1, ch.count, calls2.data(), n2.data(), o2.data(), t2.data());
    ch.z3 = seg_fill_host(2, ch.count, calls3.data(), n3.data(), o3.data(), t3.data());
    ch.seg2_off = put(t2.data(), t2.size());
    ch.seg3_off = put(t3.data(), t3.size());
    m_s2o = std::max(m_s2o, (size_t)w_s2o * 4);
    m_rh = std::max(m_rh, (size_t)w_rh * 4);
    m_f3 = std::max(m_f3, (size_t)w_f3 * 4);
    m_ct = std::max(m_ct, (size_t)w_ct * 4);
    m_samp = std::max({m_samp, seg_scratch_bytes(ch.z2), seg_scratch_bytes(ch.z3)});
  }
  // keygen over all instances: units (instance, modulus, 256 coefficients)
  {
    std::vector<uint64_t> uo(count + 1, 0);
    for (int pos = 0; pos < count; ++pos) uo[pos + 1] = uo[pos] + (uint64_t)3 * inst[pos].n / 256;
    keygen_units = (uint32_t)uo[count];
    // the keygen reads only key offsets, l, n and x: the first-chunk arena offsets are unused
    keygen_inst_off = put(inst.data(), inst.size() * sizeof(InstDev));
    keygen_unit_off = put(uo.data(), uo.size() * 8);
  }
  a_s2o = 0;
  a_rh = a_s2o + a256(m_s2o);
  a_rhsh = a_rh + a256(m_rh);
  a_f3 = a_rhsh + a256(m_rh);
  a_ct = a_f3 + a256(m_f3);
  a_samp = a_ct + a256(m_ct);
  scratch_bytes = a_samp + a256(m_samp);
  CUFE_CUDA(cudaMalloc(&tables, std::max<size_t>(blob.size(), 256)));
  CUFE_CUDA(cudaMemcpy(tables, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  if (!keys_only) {
    if (cudaMalloc(&scratch, scratch_bytes) != cudaSuccess) {
      cudaGetLastError();
      scratch = nullptr;
      set_last_error("batch: no room for " + std::to_string(scratch_bytes) + " B of step scratch");
      return CUFE_ERR_NOMEM;
    }
  }
  ran = false;
  return CUFE_OK;
}

// Times one eager step at each scratch budget (the bound buffers must be set), keeps the
// fastest layout.  A budget whose scratch does not fit the device is skipped (ms = -1).
int Batch::tune(int nb, const size_t *budgets, size_t *chosen, float *ms, cudaStream_t s) {
  if (nb < 1 || !budgets || !x || !y || !seeds2 || !seeds3 || !out) return CUFE_ERR_INVALID;
  const size_t before = chunk_budget;
  int best = -1;
  float best_ms = 0;
  for (int i = 0; i < nb; ++i) {
    if (ms) ms[i] = -1.0f;
    if (!budgets[i]) continue;
    int rc = layout(budgets[i]);
    if (rc == CUFE_ERR_NOMEM) continue;
    if (rc) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      if (e0) cudaEventDestroy(e0);
      set_last_error("batch tune: cudaEventCreate failed");
      return CUFE_ERR_CUDA;
    }
    float t = 0;
    rc = run(s);  // untimed: first use of this layout
    if (!rc && cudaEventRecord(e0, s) == cudaSuccess) rc = run(s);
    const bool ok = !rc && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
                    cudaEventElapsedTime(&t, e0, e1) == cudaSuccess;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (!ok) {
      set_last_error("batch tune: event timing failed");
      return CUFE_ERR_CUDA;
    }
    if (ms) ms[i] = t;
    if (best < 0 || t < best_ms) best = i, best_ms = t;
  }
  const int rc = layout(best >= 0 ? budgets[best] : before);
  if (rc) return rc;
  if (best < 0) {
    set_last_error("batch tune: no budget fits the device");
    return CUFE_ERR_NOMEM;
  }
  if (chosen) *chosen = budgets[best];
  return CUFE_OK;
}

void Batch::drop_graph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
}

void Batch::release() {
  drop_graph();
  if (cap) cudaStreamDestroy(cap);
  for (void *p : {(void *)keys, (void *)sky, (void *)tables, (void *)scratch, (void *)rk, (void *)perm,
                  (void *)status})
    if (p) cudaFree(p);
  keys = sky = rk = perm = status = nullptr;
  tables = scratch = nullptr;
  cap = nullptr;
  for (auto &kv : ctx) kv.second->release();
  ctx.clear();
}

int Batch::setup(const uint8_t *sa, const uint8_t *ss, const uint8_t *se, cudaStream_t s) {
  if (!sa || !se) return CUFE_ERR_INVALID;
  for (int pos = 0; pos < count; ++pos) {
    const InstDev &I = inst[pos];
    const uint32_t u = I.user;
    int rc = ctx_setup_cpu_map_l(*ctx[(int)I.n], (int)I.l, sa + 32 * (size_t)u, ss ? ss + 32 * (size_t)u : nullptr,
                                 se + 32 * (size_t)u, keys + I.mpk, keys + I.msk, s);
    if (rc) return rc;
  }
  return CUFE_OK;
}

int Batch::run(cudaStream_t s) {
  if (!x || !y || !seeds2 || !seeds3 || !out) {
    set_last_error("batch: bind the inputs and outputs first");
    return CUFE_ERR_INVALID;
  }
  if (!scratch || !tables) {  // a re-layout (cufe_batch_tune) that found no memory
    set_last_error("batch: no step scratch; re-chunk with a budget that fits");
    return CUFE_ERR_NOMEM;
  }
  uint32_t *rk2 = rk, *rk3 = rk + (size_t)count * 60;
  int rc = expand_keys_device(seeds2, perm, count, rk2, s);
  if (rc) return rc;
  rc = expand_keys_device(seeds3, perm, count, rk3, s);
  if (rc) return rc;
  {
    const size_t smem = (size_t)2 * max_l * 4;
    static bool attr = false;
    if (!attr) {
      CUFE_CUDA(cudaFuncSetAttribute(k_keygen_het, cudaFuncAttributeMaxDynamicSharedMemorySize, 32 * 1024));
      attr = true;
    }
    ProfScope ps("batch_keygen", s);
    note_launch(), k_keygen_het<<<keygen_units, 256, smem, s>>>(reinterpret_cast<const InstDev *>(tables + keygen_inst_off),
                                                 reinterpret_cast<const uint64_t *>(tables + keygen_unit_off),
                                                 (uint32_t)count, keys, y, sky, mq);
    CUFE_CUDA(cudaGetLastError());
  }
  uint32_t *s2o = reinterpret_cast<uint32_t *>(scratch + a_s2o);
  uint32_t *rh = reinterpret_cast<uint32_t *>(scratch + a_rh);
  uint32_t *rhsh = reinterpret_cast<uint32_t *>(scratch + a_rhsh);
  uint32_t *f3 = reinterpret_cast<uint32_t *>(scratch + a_f3);
  uint32_t *ct = reinterpret_cast<uint32_t *>(scratch + a_ct);
  void *samp = scratch + a_samp;
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const BatchChunk &ch = chunks[ci];
    const SegDev sg2 = seg_bind(tables + ch.seg2_off, ch.count), sg3 = seg_bind(tables + ch.seg3_off, ch.count);
    rc = sample_cpu_map_seg(1, sg2, ch.z2, rk2 + (size_t)ch.first * 60, s2o, samp, status, num_sms, s);
    if (rc) return rc;
    for (const BatchGroup &g : ch.groups) {
      const size_t nn = (size_t)1 << g.logn;
      CUFE_CUDA(cudaMemcpy2DAsync(rh + g.rh, 3 * nn * 4, s2o + g.s2o, 6 * nn * 4, 3 * nn * 4, g.count,
                                  cudaMemcpyDeviceToDevice, s));
      rc = ntt_fwd_shoup_launch(ctx[(int)nn]->ring.args, rh + g.rh, rhsh + g.rh, (long long)g.count * 3, s);
      if (rc) return rc;
    }
    rc = sample_cpu_map_seg(2, sg3, ch.z3, rk3 + (size_t)ch.first * 60, f3, samp, status, num_sms, s);
    if (rc) return rc;
    for (const BatchGroup &g : ch.groups) {
      const RingArgs &ra = ctx[1 << g.logn]->ring.args;
      rc = dispatch_logn_b(g.logn, [&](auto LL) {
        constexpr int LOGN = decltype(LL)::value;
        using P = NttPlan<LOGN>;
        constexpr int G = ppc<LOGN>();
        static bool attr = false;
        if (!attr) {
          CUFE_CUDA(cudaFuncSetAttribute(k_encrypt_het<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
          attr = true;
        }
        ProfScope ps("batch_encrypt", s);
        note_launch(), k_encrypt_het<LOGN><<<(unsigned)((g.nres + G - 1) / G), dim3(P::T, G), G * P::SMEM_WORDS * 4, s>>>(
            reinterpret_cast<const InstDev *>(tables + g.inst_off), reinterpret_cast<const uint64_t *>(tables + g.res_off),
            g.count, g.nres, keys, rh, rhsh, f3, s2o, x, ct, ra, mq);
        CUFE_CUDA(cudaGetLastError());
        return (int)CUFE_OK;
      });
      if (rc) return rc;
    }
    {
      ProfScope ps("batch_decrypt", s);
      note_launch(), k_dec_coef0_het<<<ch.count, 256, 0, s>>>(reinterpret_cast<const InstDev *>(tables + ch.inst_off), ct, sky, y,
                                              out, d0, mq, dd);
      CUFE_CUDA(cudaGetLastError());
    }
  }
  last_chunk = (int)chunks.size() - 1;
  ran = true;
  return CUFE_OK;
}

int Batch::replay(cudaStream_t s) {
  if (!exec) {
    if (!ran) {  // first-use attribute settings and workspace happen outside the capture
      int rc = run(s);
      if (rc) return rc;
      CUFE_CUDA(cudaStreamSynchronize(s));
    }
    if (!cap) CUFE_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    Prof *saved = t_prof;
    t_prof = nullptr;  // no profiling events inside the graph
    CUFE_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    const int rc = run(cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cap, &g);
    t_prof = saved;
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) {
      set_last_error(std::string("batch capture: ") + cudaGetErrorString(e));
      return CUFE_ERR_CUDA;
    }
    graph = g;
    CUFE_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  }
  CUFE_CUDA(cudaGraphLaunch(exec, s));
  return CUFE_OK;
}


// ---------------------------------------------------------------------------- serving
//
// A request server over resident tenants (a Batch holds their key pairs).  Requests:
// encrypt(tenant, x, seeds) -> a ciphertext kept in the ciphertext arena; keygen(tenant, y)
// -> a function key (and its y) kept in the key arena; decrypt(ciphertext, function key) ->
// the decoded inner product.  poll() retires finished ticks and launches the next: a tick
// admits queued requests in arrival order while its scratch, the arenas and the table
// buffer have room (admission by device-memory footprint), uploads one table blob, and runs
// encrypt (segmented sigma_2 / sigma_3 samplers, r^ NTT, per-degree encryption), keygen and
// decrypt kernels over all admitted requests.  Requests arriving while ticks run join the
// next tick; up to two ticks are in flight (one running, one queued behind it).

class WordArena {  // first-fit allocator over [0, words)
 public:
  void init(uint64_t words) {
    free_.clear();
    if (words) free_[0] = words;
    total_ = avail_ = words;
  }
  bool alloc(uint64_t w, uint64_t *off) {
    w = (w + 63) & ~63ull;  // 256-byte granules
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= w) {
        *off = it->first;
        const uint64_t rest = it->second - w, at = it->first + w;
        free_.erase(it);
        if (rest) free_[at] = rest;
        avail_ -= w;
        return true;
      }
    return false;
  }
  void release(uint64_t off, uint64_t w) {
    w = (w + 63) & ~63ull;
    auto it = free_.emplace(off, w).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
    avail_ += w;
  }
  uint64_t available() const { return avail_; }

 private:
  std::map<uint64_t, uint64_t> free_;
  uint64_t total_ = 0, avail_ = 0;
};

enum { REQ_ENCRYPT = 0, REQ_KEYGEN = 1, REQ_DECRYPT = 2 };
enum { ST_QUEUED = 0, ST_RUNNING = 1, ST_DONE = 2, ST_RELEASED = 3, ST_SHED = 4 };

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Server {
  struct Req {
    int kind = 0, tenant = 0, state = ST_QUEUED;
    std::vector<uint32_t> data;  // x (encrypt) or the bits of y (keygen)
    uint8_t s2[32], s3[32];
    int64_t ref_ct = -1, ref_sk = -1;
    uint64_t slot = 0, slot_words = 0;  // ciphertext / function-key slot
    int refs = 0;                       // decrypts not yet finished that read this slot
    bool release_pending = false;
    uint32_t value = 0;
    double t_arrival = 0, t_done = 0;
  };
  struct Tick {
    cudaEvent_t done = nullptr;
    std::vector<int64_t> ids, dec_ids;
    uint8_t *stage = nullptr;  // pinned: table blob, then the y vectors of keygens
    uint32_t *host_out = nullptr;
    bool busy = false;
  };

  Batch tenants;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<Req> reqs;
  std::deque<int64_t> queue;
  std::deque<int> inflight;  // tick indices in launch order
  Tick ticks[2];
  WordArena ct_arena, sk_arena;
  uint32_t *d_ct = nullptr, *d_sk = nullptr, *d_out = nullptr;
  uint8_t *d_tab = nullptr, *d_scr = nullptr;
  size_t tab_bytes = 0, scr_bytes = 0;
  static constexpr int kMaxDec = 65536;
  static constexpr size_t kStageY = (size_t)32 << 20;  // pinned room for a tick's keygen vectors
  uint64_t n_ticks = 0, n_done = 0, n_shed = 0;
  // overload control: requests per tick (0: memory limits only) and the longest a request may
  // wait in the queue before a tick admits it (0: forever); older requests are shed
  int max_tick_reqs = 0;
  double max_queue_s = 0;

  int create(int count, const int *n, const int *l, size_t arena_bytes, size_t tick_bytes, int dev) {
    device = dev;
    tenants.keys_only = true;  // the tenants' key pairs; ticks use the server's own scratch
    int rc = tenants.create(count, n, l, (size_t)1 << 40, dev);
    if (rc) return rc;
    if ((rc = validate(count, n, l, arena_bytes, tick_bytes))) return rc;
    if (!arena_bytes) arena_bytes = kDefaultBytes;
    if (!tick_bytes) tick_bytes = kDefaultBytes;
    tab_bytes = (size_t)64 << 20;
    scr_bytes = tick_bytes;
    CUFE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CUFE_CUDA(cudaMalloc(&d_ct, arena_bytes));
    CUFE_CUDA(cudaMalloc(&d_sk, arena_bytes / 4));
    CUFE_CUDA(cudaMalloc(&d_out, (size_t)kMaxDec * 4));
    CUFE_CUDA(cudaMalloc(&d_tab, tab_bytes));
    CUFE_CUDA(cudaMalloc(&d_scr, scr_bytes));
    ct_arena.init(arena_bytes / 4);
    sk_arena.init(arena_bytes / 16);
    for (Tick &t : ticks) {
      CUFE_CUDA(cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming));
      CUFE_CUDA(cudaMallocHost(&t.stage, tab_bytes + kStageY));
      CUFE_CUDA(cudaMallocHost(&t.host_out, (size_t)kMaxDec * 4));
    }
    return CUFE_OK;
  }

  void release_all() {
    if (stream) cudaStreamSynchronize(stream);
    for (Tick &t : ticks) {
      if (t.done) cudaEventDestroy(t.done);
      if (t.stage) cudaFreeHost(t.stage);
      if (t.host_out) cudaFreeHost(t.host_out);
      t = Tick{};
    }
    for (void *p : {(void *)d_ct, (void *)d_sk, (void *)d_out, (void *)d_tab, (void *)d_scr})
      if (p) cudaFree(p);
    d_ct = d_sk = d_out = nullptr;
    d_tab = d_scr = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    tenants.release();
  }

  const InstDev &tenant(int t) const { return tenants.inst[tenants.pos_of[t]]; }

  int64_t submit(Req &&r) {
    reqs.push_back(std::move(r));
    const int64_t id = (int64_t)reqs.size() - 1;
    Req &q = reqs.back();
    if (q.kind == REQ_DECRYPT) {
      ++reqs[q.ref_ct].refs;
      ++reqs[q.ref_sk].refs;
    }
    queue.push_back(id);
    return id;
  }

  // tick scratch available to encryptions: 1 MiB stays for alignment and the key schedules
  static uint64_t scratch_cap(uint64_t tick_bytes) { return tick_bytes > (1u << 20) ? tick_bytes - (1u << 20) : 0; }
  uint64_t scratch_cap() const { return scratch_cap(scr_bytes); }

  static constexpr size_t kDefaultBytes = (size_t)16 << 30;

  // Tenant sizes, and every request of every tenant fitting an empty tick and an empty arena
  // (a request that never fits would wait in the queue forever and block those behind it).
  // Host-only: runs before any device is touched.
  static int validate(int count, const int *n, const int *l, size_t arena_bytes, size_t tick_bytes) {
    if (count < 1 || !n || !l) return CUFE_ERR_INVALID;
    if (!arena_bytes) arena_bytes = kDefaultBytes;
    if (!tick_bytes) tick_bytes = kDefaultBytes;
    for (int t = 0; t < count; ++t) {
      if (n[t] < 256 || n[t] > 8192 || (n[t] & (n[t] - 1)) || l[t] < 1 || l[t] > 4096) {
        set_last_error("server: n must be a power of two in [256, 8192] and l in [1, 4096]");
        return CUFE_ERR_INVALID;
      }
      const uint64_t need = enc_scratch_bytes((uint32_t)n[t], (uint32_t)l[t]);
      const uint64_t ct_words = (uint64_t)(l[t] + 1) * 3 * n[t], sk_words = (uint64_t)3 * n[t] + l[t];
      if (need > scratch_cap(tick_bytes) || ct_words > arena_bytes / 4 || sk_words > arena_bytes / 16) {
        set_last_error("server: tenant " + std::to_string(t) + " (n=" + std::to_string(n[t]) +
                       ", l=" + std::to_string(l[t]) + ") needs " + std::to_string(need + (1u << 20)) +
                       " B of tick scratch and " + std::to_string(ct_words * 4) +
                       " B of ciphertext arena; tick_bytes or arena_bytes is too small");
        return CUFE_ERR_INVALID;
      }
    }
    return CUFE_OK;
  }

  static uint64_t enc_scratch_bytes(uint32_t n, uint32_t l) {
    const uint64_t poly = (uint64_t)3 * n * 4;
    const uint64_t R3 = cpu_map_refills(l, n, 2), R2 = cpu_map_refills(2, n, 1);
    // sampler scratch: 39 B per refill (candidate low words 32, accept mask 1, bit-32 and sign
    // bytes 2, prefix 4) plus tiles and call starts; 44 leaves room for the per-tile terms
    return poly * (2 + 2 + l) + std::max(R3, R2) * 44 + 2 * 60 * 4 + 8192;
  }

  void retire(Tick &t) {
    const double now = now_s();
    for (size_t k = 0; k < t.dec_ids.size(); ++k) reqs[t.dec_ids[k]].value = t.host_out[k];
    for (int64_t id : t.ids) {
      Req &r = reqs[id];
      r.state = ST_DONE;
      r.t_done = now;
      ++n_done;
      if (r.kind == REQ_DECRYPT) {
        for (int64_t ref : {r.ref_ct, r.ref_sk}) {
          Req &o = reqs[ref];
          if (--o.refs == 0 && o.release_pending) free_slot(o);
        }
      }
    }
    t.ids.clear();
    t.dec_ids.clear();
    t.busy = false;
  }

  // drop a queued request without running it; a decrypt gives back its references
  void shed(Req &r, double now) {
    r.state = ST_SHED;
    r.t_done = now;
    ++n_shed;
    if (r.kind == REQ_DECRYPT) {
      for (int64_t ref : {r.ref_ct, r.ref_sk}) {
        Req &o = reqs[ref];
        if (--o.refs == 0 && o.release_pending) free_slot(o);
      }
    }
  }

  void free_slot(Req &o) {
    if (o.state == ST_RELEASED) return;
    if (o.kind == REQ_ENCRYPT) ct_arena.release(o.slot, o.slot_words);
    if (o.kind == REQ_KEYGEN) sk_arena.release(o.slot, o.slot_words);
    o.state = ST_RELEASED;
  }

  // retire finished ticks; launch one if a tick buffer is free and work is queued
  int poll(bool wait) {
    int done0 = (int)n_done;
    while (!inflight.empty()) {
      Tick &t = ticks[inflight.front()];
      cudaError_t e = wait ? cudaEventSynchronize(t.done) : cudaEventQuery(t.done);
      if (e == cudaErrorNotReady) break;
      if (e != cudaSuccess) {
        set_last_error(std::string("server tick: ") + cudaGetErrorString(e));
        return CUFE_ERR_CUDA;
      }
      retire(t);
      inflight.pop_front();
      wait = false;
    }
    if (!queue.empty() && inflight.size() < 2) {
      const int ti = ticks[0].busy ? 1 : 0;
      int rc = launch(ti);
      if (rc) return rc;
    }
    return (int)n_done - done0;
  }

  int launch(int ti) {
    Tick &T = ticks[ti];
    // ---- admission (arrival order; a decrypt waits until its inputs were admitted)
    std::vector<int64_t> enc, kg, dec;
    uint64_t scr = 0, x_words = 0, blob_est = 1 << 16, ystage = 0;
    std::deque<int64_t> keep;
    const uint64_t scr_cap = scratch_cap();
    const double now = now_s();
    while (!queue.empty()) {
      if (max_tick_reqs > 0 && enc.size() + kg.size() + dec.size() >= (size_t)max_tick_reqs) break;
      const int64_t id = queue.front();
      queue.pop_front();
      Req &r = reqs[id];
      if ((max_queue_s > 0 && now - r.t_arrival > max_queue_s) ||
          (r.kind == REQ_DECRYPT && (reqs[r.ref_ct].state == ST_SHED || reqs[r.ref_sk].state == ST_SHED))) {
        shed(r, now);
        continue;
      }
      const InstDev &I = tenant(r.tenant);
      bool ok = true;
      if (r.kind == REQ_ENCRYPT) {
        const uint64_t need = enc_scratch_bytes(I.n, I.l), tab = 2 * sizeof(InstDev) + 512 + 4ull * I.l;
        ok = scr + need <= scr_cap && blob_est + tab <= tab_bytes && enc.size() < 4096 &&
             ct_arena.alloc((uint64_t)(I.l + 1) * 3 * I.n, &r.slot);
        if (ok) {
          r.slot_words = (uint64_t)(I.l + 1) * 3 * I.n;
          scr += need;
          blob_est += tab;
          x_words += I.l;
          enc.push_back(id);
        }
      } else if (r.kind == REQ_KEYGEN) {
        const uint64_t yb = a256(4ull * I.l);
        ok = kg.size() < 4096 && ystage + yb <= kStageY && blob_est + 2 * sizeof(InstDev) <= tab_bytes &&
             sk_arena.alloc((uint64_t)3 * I.n + I.l, &r.slot);
        if (ok) {
          r.slot_words = (uint64_t)3 * I.n + I.l;
          ystage += yb;
          blob_est += 2 * sizeof(InstDev);
          kg.push_back(id);
        }
      } else {
        ok = dec.size() < (size_t)kMaxDec && blob_est + sizeof(InstDev) <= tab_bytes &&
             reqs[r.ref_ct].state != ST_QUEUED && reqs[r.ref_sk].state != ST_QUEUED;
        if (ok) {
          blob_est += sizeof(InstDev);
          dec.push_back(id);
        }
      }
      if (ok) {
        r.state = ST_RUNNING;
      } else {
        keep.push_back(id);
        if (r.kind == REQ_ENCRYPT && scr + enc_scratch_bytes(I.n, I.l) > scr_cap) break;  // tick full
      }
    }
    while (!keep.empty()) {
      queue.push_front(keep.back());
      keep.pop_back();
    }
    if (enc.empty() && kg.empty() && dec.empty()) return CUFE_OK;
    // ---- tables: encryptions grouped by ring degree
    std::stable_sort(enc.begin(), enc.end(),
                     [&](int64_t a, int64_t b) { return tenant(reqs[a].tenant).n < tenant(reqs[b].tenant).n; });
    std::vector<uint8_t> blob;
    auto put = [&](const void *src, size_t bytes) {
      const size_t off = a256(blob.size());
      blob.resize(off + a256(bytes));
      if (src && bytes) std::memcpy(blob.data() + off, src, bytes);
      return off;
    };
    const uint32_t ne = (uint32_t)enc.size();
    std::vector<InstDev> ei(ne);
    std::vector<uint32_t> calls2(ne, 2), nn(ne), calls3(ne);
    std::vector<uint64_t> o2(ne), o3(ne);
    uint64_t w_s2o = 0, w_rh = 0, w_f3 = 0, w_x = 0;
    std::vector<BatchGroup> groups;
    std::vector<uint32_t> xs;
    xs.reserve(x_words);
    for (uint32_t k = 0; k < ne; ++k) {
      const Req &r = reqs[enc[k]];
      InstDev I = tenant(r.tenant);
      const int logn = __builtin_ctz(I.n);
      if (groups.empty() || groups.back().logn != logn) {
        BatchGroup g;
        g.logn = logn;
        g.first = k;
        g.rh = w_rh;
        g.s2o = w_s2o;
        groups.push_back(g);
      }
      ++groups.back().count;
      groups.back().nres += (long long)(I.l + 1) * 3;
      I.ct = r.slot;
      I.s2o = w_s2o;
      I.rh = w_rh;
      I.f3 = w_f3;
      I.x = w_x;
      xs.insert(xs.end(), r.data.begin(), r.data.end());
      nn[k] = I.n;
      calls3[k] = I.l;
      o2[k] = w_s2o;
      o3[k] = w_f3;
      w_s2o += (uint64_t)6 * I.n;
      w_rh += (uint64_t)3 * I.n;
      w_f3 += (uint64_t)I.l * 3 * I.n;
      w_x += I.l;
      ei[k] = I;
    }
    SegSizes z2{}, z3{};
    size_t seg2 = 0, seg3 = 0, x_off = 0, seeds_off = 0;
    for (BatchGroup &g : groups) {
      g.inst_off = put(ei.data() + g.first, (size_t)g.count * sizeof(InstDev));
      std::vector<uint64_t> ro(g.count + 1, 0);
      for (uint32_t k = 0; k < g.count; ++k) ro[k + 1] = ro[k] + (uint64_t)(ei[g.first + k].l + 1) * 3;
      g.res_off = put(ro.data(), ro.size() * 8);
    }
    if (ne) {
      std::vector<uint8_t> t2(seg_layout(ne).bytes), t3(seg_layout(ne).bytes);
      z2 = seg_fill_host(1, ne, calls2.data(), nn.data(), o2.data(), t2.data());
      z3 = seg_fill_host(2, ne, calls3.data(), nn.data(), o3.data(), t3.data());
      seg2 = put(t2.data(), t2.size());
      seg3 = put(t3.data(), t3.size());
      x_off = put(xs.data(), xs.size() * 4);
      std::vector<uint8_t> sd((size_t)2 * ne * 32);
      for (uint32_t k = 0; k < ne; ++k) {
        std::memcpy(sd.data() + 32 * (size_t)k, reqs[enc[k]].s2, 32);
        std::memcpy(sd.data() + 32 * (size_t)(ne + k), reqs[enc[k]].s3, 32);
      }
      seeds_off = put(sd.data(), sd.size());
    }
    // keygen: y lives in the function-key slot after its 3n words
    std::vector<InstDev> ki(kg.size());
    std::vector<uint64_t> uo(kg.size() + 1, 0);
    for (size_t k = 0; k < kg.size(); ++k) {
      const Req &r = reqs[kg[k]];
      InstDev I = tenant(r.tenant);
      I.sky = r.slot;
      I.x = r.slot + (uint64_t)3 * I.n;
      ki[k] = I;
      uo[k + 1] = uo[k] + (uint64_t)3 * I.n / 256;
    }
    uint32_t max_l = 1;
    for (const InstDev &I : ki) max_l = std::max(max_l, I.l);
    const size_t kg_inst = put(ki.data(), ki.size() * sizeof(InstDev)), kg_units = put(uo.data(), uo.size() * 8);
    // decrypt: ciphertext slot, function-key slot and its y
    std::vector<InstDev> di(dec.size());
    for (size_t k = 0; k < dec.size(); ++k) {
      const Req &r = reqs[dec[k]];
      const Req &c = reqs[r.ref_ct], &f = reqs[r.ref_sk];
      InstDev I = tenant(c.tenant);
      I.ct = c.slot;
      I.sky = f.slot;
      I.x = f.slot + (uint64_t)3 * I.n;
      I.user = (uint32_t)k;
      di[k] = I;
    }
    const size_t dec_inst = put(di.data(), di.size() * sizeof(InstDev));
    if (blob.size() > tab_bytes) {  // cannot happen with the admission limits; refuse loudly
      set_last_error("server: tick tables exceed the table buffer");
      return CUFE_ERR_INVALID;
    }
    // ---- upload and launch (all on the server stream)
    std::memcpy(T.stage, blob.data(), blob.size());
    CUFE_CUDA(cudaMemcpyAsync(d_tab, T.stage, blob.size(), cudaMemcpyHostToDevice, stream));
    size_t ys = a256(blob.size());
    for (size_t k = 0; k < kg.size(); ++k) {
      const Req &r = reqs[kg[k]];
      std::memcpy(T.stage + ys, r.data.data(), r.data.size() * 4);
      CUFE_CUDA(cudaMemcpyAsync(d_sk + ki[k].x, T.stage + ys, r.data.size() * 4, cudaMemcpyHostToDevice, stream));
      ys += a256(r.data.size() * 4);
    }
    int rc = CUFE_OK;
    if (ne) {
      // scratch: s2o | rh | rh_sh | f3 | round keys | sampler scratch
      uint8_t *p = d_scr;
      auto take = [&](size_t b) {
        uint8_t *q = p;
        p += a256(b);
        return q;
      };
      uint32_t *s2o = reinterpret_cast<uint32_t *>(take(w_s2o * 4));
      uint32_t *rh = reinterpret_cast<uint32_t *>(take(w_rh * 4));
      uint32_t *rhsh = reinterpret_cast<uint32_t *>(take(w_rh * 4));
      uint32_t *f3 = reinterpret_cast<uint32_t *>(take(w_f3 * 4));
      uint32_t *rk = reinterpret_cast<uint32_t *>(take((size_t)2 * ne * 60 * 4));
      const size_t before = (size_t)(p - d_scr);
      if (before + std::max(seg_scratch_bytes(z2), seg_scratch_bytes(z3)) > scr_bytes)
        z2.doubling = z3.doubling = false;  // no room for the doubling tables: serial walk
      void *samp = take(std::max(seg_scratch_bytes(z2), seg_scratch_bytes(z3)));
      if ((size_t)(p - d_scr) > scr_bytes) {
        set_last_error("server: tick scratch exceeded");
        return CUFE_ERR_INVALID;
      }
      const uint8_t *seeds = d_tab + seeds_off;
      if ((rc = expand_keys_device(seeds, nullptr, 2 * ne, rk, stream))) return rc;
      if ((rc = sample_cpu_map_seg(1, seg_bind(d_tab + seg2, ne), z2, rk, s2o, samp, tenants.status, tenants.num_sms,
                                   stream)))
        return rc;
      for (const BatchGroup &g : groups) {
        const size_t nn1 = (size_t)1 << g.logn;
        CUFE_CUDA(cudaMemcpy2DAsync(rh + g.rh, 3 * nn1 * 4, s2o + g.s2o, 6 * nn1 * 4, 3 * nn1 * 4, g.count,
                                    cudaMemcpyDeviceToDevice, stream));
        if ((rc = ntt_fwd_shoup_launch(tenants.ctx[(int)nn1]->ring.args, rh + g.rh, rhsh + g.rh,
                                       (long long)g.count * 3, stream)))
          return rc;
      }
      if ((rc = sample_cpu_map_seg(2, seg_bind(d_tab + seg3, ne), z3, rk + (size_t)ne * 60, f3, samp, tenants.status,
                                   tenants.num_sms, stream)))
        return rc;
      const uint32_t *xd = reinterpret_cast<const uint32_t *>(d_tab + x_off);
      for (const BatchGroup &g : groups) {
        const RingArgs &ra = tenants.ctx[1 << g.logn]->ring.args;
        rc = dispatch_logn_b(g.logn, [&](auto LL) {
          constexpr int LOGN = decltype(LL)::value;
          using P = NttPlan<LOGN>;
          constexpr int G = ppc<LOGN>();
          static bool attr = false;
          if (!attr) {
            CUFE_CUDA(cudaFuncSetAttribute(k_encrypt_het<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
            attr = true;
          }
          ProfScope ps("serve_encrypt", stream);
          note_launch(), k_encrypt_het<LOGN><<<(unsigned)((g.nres + G - 1) / G), dim3(P::T, G), G * P::SMEM_WORDS * 4, stream>>>(
              reinterpret_cast<const InstDev *>(d_tab + g.inst_off), reinterpret_cast<const uint64_t *>(d_tab + g.res_off),
              g.count, g.nres, tenants.keys, rh, rhsh, f3, s2o, xd, d_ct, ra, tenants.mq);
          CUFE_CUDA(cudaGetLastError());
          return (int)CUFE_OK;
        });
        if (rc) return rc;
      }
    }
    if (!kg.empty()) {
      static bool attr = false;
      if (!attr) {
        CUFE_CUDA(cudaFuncSetAttribute(k_keygen_het, cudaFuncAttributeMaxDynamicSharedMemorySize, 32 * 1024));
        attr = true;
      }
      ProfScope ps("serve_keygen", stream);
      note_launch(), k_keygen_het<<<(unsigned)uo.back(), 256, (size_t)2 * max_l * 4, stream>>>(
          reinterpret_cast<const InstDev *>(d_tab + kg_inst), reinterpret_cast<const uint64_t *>(d_tab + kg_units),
          (uint32_t)kg.size(), tenants.keys, reinterpret_cast<const int32_t *>(d_sk), d_sk, tenants.mq);
      CUFE_CUDA(cudaGetLastError());
    }
    if (!dec.empty()) {
      ProfScope ps("serve_decrypt", stream);
      note_launch(), k_dec_coef0_het<<<(unsigned)dec.size(), 256, 0, stream>>>(reinterpret_cast<const InstDev *>(d_tab + dec_inst),
                                                               d_ct, d_sk, reinterpret_cast<const int32_t *>(d_sk),
                                                               d_out, nullptr, tenants.mq, tenants.dd);
      CUFE_CUDA(cudaGetLastError());
      CUFE_CUDA(cudaMemcpyAsync(T.host_out, d_out, dec.size() * 4, cudaMemcpyDeviceToHost, stream));
    }
    CUFE_CUDA(cudaEventRecord(T.done, stream));
    T.ids = enc;
    T.ids.insert(T.ids.end(), kg.begin(), kg.end());
    T.ids.insert(T.ids.end(), dec.begin(), dec.end());
    T.dec_ids = dec;
    T.busy = true;
    inflight.push_back((int)(&T - ticks));
    ++n_ticks;
    return CUFE_OK;
  }
};

}  // namespace cufe

// ---------------------------------------------------------------------------- C ABI

struct cufe_batch {
  cufe::Batch b;
  std::mutex mu;
  cufe::Prof prof;  // eager steps' kernel timing (cufe_batch_profile)
};

extern "C" {

int cufe_batch_create(cufe_batch **out, int count, const int *n, const int *l, size_t max_chunk_bytes, int device) {
  if (!out) return CUFE_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cufe::set_last_error("no CUDA device");
    return CUFE_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return CUFE_ERR_INVALID;
  cufe_batch *h = new cufe_batch;
  const int rc = h->b.create(count, n, l, max_chunk_bytes, device);
  if (rc) {
    h->b.release();
    delete h;
    return rc;
  }
  *out = h;
  return CUFE_OK;
}

int cufe_batch_destroy(cufe_batch *h) {
  if (!h) return CUFE_ERR_INVALID;
  cudaSetDevice(h->b.device);
  h->b.release();
  delete h;
  return CUFE_OK;
}

int cufe_batch_setup(cufe_batch *h, const uint8_t *seeds_a, const uint8_t *seeds_s, const uint8_t *seeds_e,
                     void *stream) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (cudaSetDevice(h->b.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return h->b.setup(seeds_a, seeds_s, seeds_e, static_cast<cudaStream_t>(stream));
}

int cufe_batch_bind(cufe_batch *h, const uint32_t *d_x, const int32_t *d_y, const uint8_t *d_seeds2,
                    const uint8_t *d_seeds3, uint32_t *d_out, uint32_t *d_d0) {
  if (!h || !d_x || !d_y || !d_seeds2 || !d_seeds3 || !d_out) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  cufe::Batch &b = h->b;
  if (b.x != d_x || b.y != d_y || b.seeds2 != d_seeds2 || b.seeds3 != d_seeds3 || b.out != d_out || b.d0 != d_d0)
    b.drop_graph();
  b.x = d_x;
  b.y = d_y;
  b.seeds2 = d_seeds2;
  b.seeds3 = d_seeds3;
  b.out = d_out;
  b.d0 = d_d0;
  return CUFE_OK;
}

int cufe_batch_run(cufe_batch *h, void *stream) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (cudaSetDevice(h->b.device) != cudaSuccess) return CUFE_ERR_CUDA;
  cufe::t_prof = &h->prof;
  const int rc = h->b.run(static_cast<cudaStream_t>(stream));
  cufe::t_prof = nullptr;
  return rc;
}

int cufe_batch_tune(cufe_batch *h, int ncand, const size_t *budgets, size_t *chosen, float *ms, void *stream) {
  if (!h || h->b.keys_only) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (cudaSetDevice(h->b.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return h->b.tune(ncand, budgets, chosen, ms, static_cast<cudaStream_t>(stream));
}

int cufe_batch_profile(cufe_batch *h, int on) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  h->prof.collect();
  h->prof.acc.clear();
  h->prof.kernels = 0;
  h->prof.on = on != 0;
  return CUFE_OK;
}

int cufe_batch_profile_read(cufe_batch *h, double *kernel_ms, long long *kernels) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  h->prof.collect();
  double ms = 0;
  long long k = 0;
  for (const auto &kv : h->prof.acc) {
    ms += kv.second.second;
    k += kv.second.first;
  }
  if (kernel_ms) *kernel_ms = ms;
  if (kernels) *kernels = k;
  return CUFE_OK;
}

int cufe_batch_profile_groups(cufe_batch *h, int max_groups, char *names, long long *launches, double *ms) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  h->prof.collect();
  int i = 0;
  for (const auto &kv : h->prof.acc) {
    if (i >= max_groups) break;
    if (names) {
      std::strncpy(names + 64 * (size_t)i, kv.first.c_str(), 63);
      names[64 * (size_t)i + 63] = 0;
    }
    if (launches) launches[i] = kv.second.first;
    if (ms) ms[i] = kv.second.second;
    ++i;
  }
  return i;
}

int cufe_batch_graph_kernels(cufe_batch *h) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->b.graph) return 0;
  size_t nodes = 0;
  if (cudaGraphGetNodes(h->b.graph, nullptr, &nodes) != cudaSuccess) return CUFE_ERR_CUDA;
  std::vector<cudaGraphNode_t> v(nodes);
  if (nodes && cudaGraphGetNodes(h->b.graph, v.data(), &nodes) != cudaSuccess) return CUFE_ERR_CUDA;
  int kernels = 0;
  for (cudaGraphNode_t nd : v) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) return CUFE_ERR_CUDA;
    kernels += t == cudaGraphNodeTypeKernel;
  }
  return kernels;
}

int cufe_batch_replay(cufe_batch *h, void *stream) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (cudaSetDevice(h->b.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return h->b.replay(static_cast<cudaStream_t>(stream));
}

int cufe_batch_status(cufe_batch *h) {
  if (!h) return CUFE_ERR_INVALID;
  uint32_t st = 0;
  if (cudaSetDevice(h->b.device) != cudaSuccess || cudaMemcpy(&st, h->b.status, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return CUFE_ERR_CUDA;
  if (st) {
    cufe::set_last_error("batch: sampler status " + std::to_string(st));
    return CUFE_ERR_SAMPLER;
  }
  return CUFE_OK;
}

int cufe_batch_info(const cufe_batch *h, uint64_t *x_off, int *chunks, size_t *key_bytes, size_t *scratch_bytes) {
  if (!h) return CUFE_ERR_INVALID;
  const cufe::Batch &b = h->b;
  if (x_off) std::copy(b.x_off.begin(), b.x_off.end(), x_off);
  if (chunks) *chunks = (int)b.chunks.size();
  if (key_bytes) *key_bytes = b.key_bytes;
  if (scratch_bytes) *scratch_bytes = b.scratch_bytes;
  return CUFE_OK;
}

int cufe_batch_instance(const cufe_batch *h, int i, const uint32_t **mpk, const uint32_t **msk, const uint32_t **sky,
                        const uint32_t **ct) {
  if (!h || i < 0 || i >= h->b.count) return CUFE_ERR_INVALID;
  const cufe::Batch &b = h->b;
  int pos = -1;
  for (int k = 0; k < b.count; ++k)
    if ((int)b.inst[k].user == i) pos = k;
  const cufe::InstDev &I = b.inst[pos];
  if (mpk) *mpk = b.keys + I.mpk;
  if (msk) *msk = b.keys + I.msk;
  if (sky) *sky = b.sky + I.sky;
  if (ct) *ct = (b.chunks.size() == 1 && b.ran)
                    ? reinterpret_cast<const uint32_t *>(b.scratch + b.a_ct) + I.ct
                    : nullptr;
  return CUFE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------- server C ABI

struct cufe_server {
  cufe::Server s;
  std::mutex mu;
};

extern "C" {

double cufe_server_now(void) { return cufe::now_s(); }

int cufe_server_create(cufe_server **out, int tenants, const int *n, const int *l, size_t arena_bytes,
                       size_t tick_bytes, int device) {
  if (!out) return CUFE_ERR_INVALID;
  *out = nullptr;
  if (int rc = cufe::Server::validate(tenants, n, l, arena_bytes, tick_bytes)) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cufe::set_last_error("no CUDA device");
    return CUFE_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return CUFE_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return CUFE_ERR_CUDA;
  cufe_server *h = new cufe_server;
  const int rc = h->s.create(tenants, n, l, arena_bytes, tick_bytes, device);
  if (rc) {
    h->s.release_all();
    delete h;
    return rc;
  }
  *out = h;
  return CUFE_OK;
}

int cufe_server_destroy(cufe_server *h) {
  if (!h) return CUFE_ERR_INVALID;
  cudaSetDevice(h->s.device);
  h->s.release_all();
  delete h;
  return CUFE_OK;
}

int cufe_server_setup(cufe_server *h, const uint8_t *seeds_a, const uint8_t *seeds_s, const uint8_t *seeds_e) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (cudaSetDevice(h->s.device) != cudaSuccess) return CUFE_ERR_CUDA;
  int rc = h->s.tenants.setup(seeds_a, seeds_s, seeds_e, h->s.stream);
  if (rc) return rc;
  CUFE_CUDA(cudaStreamSynchronize(h->s.stream));
  return CUFE_OK;
}

long long cufe_server_encrypt(cufe_server *h, int tenant, const uint32_t *x, const uint8_t *seed2,
                              const uint8_t *seed3, double t_arrival) {
  if (!h || !x || !seed2 || !seed3 || tenant < 0 || tenant >= h->s.tenants.count) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  cufe::Server::Req r;
  r.kind = cufe::REQ_ENCRYPT;
  r.tenant = tenant;
  r.data.assign(x, x + h->s.tenants.l[tenant]);
  std::memcpy(r.s2, seed2, 32);
  std::memcpy(r.s3, seed3, 32);
  r.t_arrival = t_arrival >= 0 ? t_arrival : cufe::now_s();
  return h->s.submit(std::move(r));
}

long long cufe_server_keygen(cufe_server *h, int tenant, const int32_t *y, double t_arrival) {
  if (!h || !y || tenant < 0 || tenant >= h->s.tenants.count) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  cufe::Server::Req r;
  r.kind = cufe::REQ_KEYGEN;
  r.tenant = tenant;
  r.data.assign(reinterpret_cast<const uint32_t *>(y), reinterpret_cast<const uint32_t *>(y) + h->s.tenants.l[tenant]);
  r.t_arrival = t_arrival >= 0 ? t_arrival : cufe::now_s();
  return h->s.submit(std::move(r));
}

long long cufe_server_decrypt(cufe_server *h, long long ct, long long sk, double t_arrival) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  auto &R = h->s.reqs;
  if (ct < 0 || sk < 0 || ct >= (long long)R.size() || sk >= (long long)R.size() ||
      R[ct].kind != cufe::REQ_ENCRYPT || R[sk].kind != cufe::REQ_KEYGEN || R[ct].tenant != R[sk].tenant ||
      R[ct].state == cufe::ST_RELEASED || R[sk].state == cufe::ST_RELEASED || R[ct].state == cufe::ST_SHED ||
      R[sk].state == cufe::ST_SHED || R[ct].release_pending ||
      R[sk].release_pending) {
    cufe::set_last_error("decrypt: needs a live ciphertext and function key of the same tenant");
    return CUFE_ERR_INVALID;
  }
  cufe::Server::Req r;
  r.kind = cufe::REQ_DECRYPT;
  r.tenant = R[ct].tenant;
  r.ref_ct = ct;
  r.ref_sk = sk;
  r.t_arrival = t_arrival >= 0 ? t_arrival : cufe::now_s();
  return h->s.submit(std::move(r));
}

int cufe_server_poll(cufe_server *h, int wait) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (cudaSetDevice(h->s.device) != cudaSuccess) return CUFE_ERR_CUDA;
  return h->s.poll(wait != 0);
}

int cufe_server_pending(cufe_server *h, long long *queued, int *ticks_in_flight) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (queued) *queued = (long long)h->s.queue.size();
  if (ticks_in_flight) *ticks_in_flight = (int)h->s.inflight.size();
  return CUFE_OK;
}

int cufe_server_result(cufe_server *h, long long id, int *state, uint32_t *value, double *t_arrival, double *t_done) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (id < 0 || id >= (long long)h->s.reqs.size()) return CUFE_ERR_INVALID;
  const auto &r = h->s.reqs[id];
  if (state) *state = r.state;
  if (value) *value = r.value;
  if (t_arrival) *t_arrival = r.t_arrival;
  if (t_done) *t_done = r.t_done;
  return CUFE_OK;
}

int cufe_server_read(cufe_server *h, long long id, uint32_t *host, size_t words) {
  if (!h || !host) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (id < 0 || id >= (long long)h->s.reqs.size()) return CUFE_ERR_INVALID;
  const auto &r = h->s.reqs[id];
  if (r.state != cufe::ST_DONE || r.kind == cufe::REQ_DECRYPT || words > r.slot_words) return CUFE_ERR_INVALID;
  const uint32_t *src = (r.kind == cufe::REQ_ENCRYPT ? h->s.d_ct : h->s.d_sk) + r.slot;
  if (cudaSetDevice(h->s.device) != cudaSuccess) return CUFE_ERR_CUDA;
  CUFE_CUDA(cudaMemcpy(host, src, words * 4, cudaMemcpyDeviceToHost));
  return CUFE_OK;
}

int cufe_server_release(cufe_server *h, long long id) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (id < 0 || id >= (long long)h->s.reqs.size()) return CUFE_ERR_INVALID;
  auto &r = h->s.reqs[id];
  if (r.kind == cufe::REQ_DECRYPT || r.state != cufe::ST_DONE) return CUFE_ERR_INVALID;
  r.release_pending = true;
  if (r.refs == 0) h->s.free_slot(r);
  return CUFE_OK;
}

int cufe_server_limits(cufe_server *h, int max_tick_requests, double max_queue_seconds) {
  if (!h || max_tick_requests < 0 || !(max_queue_seconds >= 0)) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  h->s.max_tick_reqs = max_tick_requests;
  h->s.max_queue_s = max_queue_seconds;
  return CUFE_OK;
}

long long cufe_server_shed(cufe_server *h) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  return (long long)h->s.n_shed;
}

int cufe_server_stats(cufe_server *h, long long *ticks, long long *done, size_t *ct_free_bytes) {
  if (!h) return CUFE_ERR_INVALID;
  std::lock_guard<std::mutex> g(h->mu);
  if (ticks) *ticks = (long long)h->s.n_ticks;
  if (done) *done = (long long)h->s.n_done;
  if (ct_free_bytes) *ct_free_bytes = (size_t)h->s.ct_arena.available() * 4;
  return CUFE_OK;
}

}  // extern "C"
