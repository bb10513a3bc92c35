// serial.cu -- serialized keys and ciphertexts.
//
// Format (little-endian): a 32-byte header
//   magic "CUFE" | version u16 = 1 | kind u16 | n u32 | l u32 | count u32 | polys u32 |
//   payload bytes u64
// then, for each of `count` objects and each of its `polys` residue polynomials (modulus
// r mod 3 for polynomial r, the layout of src/rlwe_sife.h:10-26), the n canonical residues
// packed LSB-first at the bit width of the modulus -- 24 bits for q_0 < 2^24, 31 bits for
// q_1, q_2 < 2^31 -- each polynomial padded to a whole 32-bit word.  86 bits per coefficient
// triple instead of 96.  Unpacking rejects any residue >= its modulus.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "ctx.h"
#include "prof.h"
#include "sampler_host.h"

namespace cufe {

namespace {

constexpr uint32_t kMagic = 0x45465543u;  // "CUFE"

struct Header {
  uint32_t magic;
  uint16_t version, kind;
  uint32_t n, l, count, polys;
  uint64_t payload;
};
static_assert(sizeof(Header) == 32, "header layout");

__host__ __device__ inline uint64_t poly_words(uint32_t n, int width) { return ((uint64_t)n * width + 31) / 32; }

// words of one object: per residue polynomial r, modulus r % 3
__host__ __device__ inline uint64_t object_words(uint32_t n, uint32_t polys) {
  const uint64_t triple = poly_words(n, 24) + 2 * poly_words(n, 31);
  return (polys / 3) * triple + (polys % 3 > 0 ? poly_words(n, 24) : 0) + (polys % 3 > 1 ? poly_words(n, 31) : 0);
}
__host__ __device__ inline uint64_t poly_offset(uint32_t n, uint32_t r) {
  return (uint64_t)(r / 3) * (poly_words(n, 24) + 2 * poly_words(n, 31)) +
         (r % 3 > 0 ? poly_words(n, 24) : 0) + (r % 3 > 1 ? poly_words(n, 31) : 0);
}

// one thread per 32 residues of one polynomial: 32 x width bits = width words
__global__ void k_pack(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, uint32_t n, uint32_t polys,
                       uint64_t groups, uint32_t q0, uint32_t q1, uint32_t q2) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gpp = (n + 31) / 32;  // groups per polynomial
  if (gid >= groups) return;
  const uint64_t poly = gid / gpp;
  const uint32_t grp = (uint32_t)(gid - poly * gpp), r = (uint32_t)(poly % polys);
  const uint64_t obj = poly / polys;
  const int m = (int)(r % 3), w = m == 0 ? 24 : 31;
  const uint32_t q = m == 0 ? q0 : (m == 1 ? q1 : q2);
  const uint32_t *s = src + poly * n + (uint64_t)grp * 32;
  uint32_t *d = dst + obj * object_words(n, polys) + poly_offset(n, r);
  const uint32_t cnt = min(32u, n - grp * 32);
  uint64_t acc = 0;
  int bits = 0;
  uint64_t wo = ((uint64_t)grp * 32 * w) / 32;  // first output word (32-value groups are word aligned)
  for (uint32_t i = 0; i < cnt; ++i) {
    acc |= (uint64_t)(s[i] % q) << bits;
    bits += w;
    if (bits >= 32) {
      d[wo++] = (uint32_t)acc;
      acc >>= 32;
      bits -= 32;
    }
  }
  if (bits > 0) d[wo] = (uint32_t)acc;
}

__global__ void k_unpack(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, uint32_t n, uint32_t polys,
                         uint64_t groups, uint32_t q0, uint32_t q1, uint32_t q2, uint32_t *__restrict__ bad) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gpp = (n + 31) / 32;
  if (gid >= groups) return;
  const uint64_t poly = gid / gpp;
  const uint32_t grp = (uint32_t)(gid - poly * gpp), r = (uint32_t)(poly % polys);
  const uint64_t obj = poly / polys;
  const int m = (int)(r % 3), w = m == 0 ? 24 : 31;
  const uint32_t q = m == 0 ? q0 : (m == 1 ? q1 : q2), mask = (1u << w) - 1u;
  const uint32_t *s = src + obj * object_words(n, polys) + poly_offset(n, r);
  uint32_t *d = dst + poly * n + (uint64_t)grp * 32;
  const uint32_t cnt = min(32u, n - grp * 32);
  uint64_t wi = ((uint64_t)grp * 32 * w) / 32;
  uint64_t acc = s[wi++];
  int bits = 32;
  uint32_t err = 0;
  for (uint32_t i = 0; i < cnt; ++i) {
    if (bits < w) {
      acc |= (uint64_t)s[wi++] << bits;
      bits += 32;
    }
    const uint32_t v = (uint32_t)acc & mask;
    acc >>= w;
    bits -= w;
    err |= v >= q;
    d[i] = v;
  }
  if (err) atomicOr(bad, 1u);
}

uint32_t kind_polys(int kind, int l) {
  switch (kind) {
    case CUFE_OBJ_MPK: return (uint32_t)(l + 1) * 3;
    case CUFE_OBJ_MSK: return (uint32_t)l * 3;
    case CUFE_OBJ_CT: return (uint32_t)(l + 1) * 3;
    case CUFE_OBJ_SKY: return 3;
    case CUFE_OBJ_DY: return 3;
  }
  return 0;
}

}  // namespace

long long serialized_bytes(const Ctx &c, int kind, int count) {
  const uint32_t polys = kind_polys(kind, c.l);
  if (!polys || count < 1) return CUFE_ERR_INVALID;
  return (long long)(sizeof(Header) + object_words(c.n, polys) * 4 * (uint64_t)count);
}

int ctx_serialize(Ctx &c, int kind, int count, const uint32_t *d_src, uint8_t *d_dst, cudaStream_t s) {
  const long long bytes = serialized_bytes(c, kind, count);
  if (bytes < 0 || !d_src || !d_dst) return CUFE_ERR_INVALID;
  if (reinterpret_cast<uintptr_t>(d_dst) % 4) {
    set_last_error("serialize: the destination must be 4-byte aligned");
    return CUFE_ERR_INVALID;
  }
  const uint32_t polys = kind_polys(kind, c.l);
  Header h{kMagic, 1, (uint16_t)kind, (uint32_t)c.n, (uint32_t)c.l, (uint32_t)count, polys,
           (uint64_t)bytes - sizeof(Header)};
  CUFE_CUDA(cudaMemcpyAsync(d_dst, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  CUFE_CUDA(cudaMemsetAsync(d_dst + sizeof(h), 0, (size_t)h.payload, s));
  const uint64_t groups = (uint64_t)count * polys * ((c.n + 31) / 32);
  ProfScope ps("serialize", s);
  note_launch(), k_pack<<<(unsigned)((groups + 255) / 256), 256, 0, s>>>(d_src, reinterpret_cast<uint32_t *>(d_dst + sizeof(h)),
                                                         (uint32_t)c.n, polys, groups, kRefPrimes[0], kRefPrimes[1],
                                                         kRefPrimes[2]);
  CUFE_CUDA(cudaGetLastError());
  // the header copy reads a host local: finish it before returning
  CUFE_CUDA(cudaStreamSynchronize(s));
  return CUFE_OK;
}

int ctx_deserialize(Ctx &c, int kind, int count, const uint8_t *d_src, size_t src_bytes, uint32_t *d_dst,
                    cudaStream_t s) {
  const long long bytes = serialized_bytes(c, kind, count);
  if (bytes < 0 || !d_src || !d_dst) return CUFE_ERR_INVALID;
  if ((long long)src_bytes < bytes || reinterpret_cast<uintptr_t>(d_src) % 4) {
    set_last_error("deserialize: buffer shorter than the object or not 4-byte aligned");
    return CUFE_ERR_INVALID;
  }
  Header h;
  CUFE_CUDA(cudaMemcpyAsync(&h, d_src, sizeof(h), cudaMemcpyDeviceToHost, s));
  CUFE_CUDA(cudaStreamSynchronize(s));
  const uint32_t polys = kind_polys(kind, c.l);
  if (h.magic != kMagic || h.version != 1 || h.kind != kind || h.n != (uint32_t)c.n || h.l != (uint32_t)c.l ||
      h.count != (uint32_t)count || h.polys != polys || h.payload != (uint64_t)bytes - sizeof(Header)) {
    set_last_error("deserialize: header does not describe this object (magic, version, kind, n, l, count)");
    return CUFE_ERR_INVALID;
  }
  int rc = c.ensure_ws(256);
  if (rc) return rc;
  uint32_t *bad = reinterpret_cast<uint32_t *>(c.ws);
  CUFE_CUDA(cudaMemsetAsync(bad, 0, 4, s));
  const uint64_t groups = (uint64_t)count * polys * ((c.n + 31) / 32);
  {
    ProfScope ps("deserialize", s);
    note_launch(), k_unpack<<<(unsigned)((groups + 255) / 256), 256, 0, s>>>(reinterpret_cast<const uint32_t *>(d_src + sizeof(h)),
                                                             d_dst, (uint32_t)c.n, polys, groups, kRefPrimes[0],
                                                             kRefPrimes[1], kRefPrimes[2], bad);
  }
  CUFE_CUDA(cudaGetLastError());
  uint32_t flag = 0;
  CUFE_CUDA(cudaMemcpyAsync(&flag, bad, 4, cudaMemcpyDeviceToHost, s));
  CUFE_CUDA(cudaStreamSynchronize(s));
  if (flag) {
    set_last_error("deserialize: a residue is not below its modulus");
    return CUFE_ERR_INVALID;
  }
  return CUFE_OK;
}

}  // namespace cufe
