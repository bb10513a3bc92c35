// sampler_host.h -- host entry points of the sampler kernels (sampler.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>

namespace cufe {

// the params.h RNS primes q_j = 2^k1 - 2^k2 + 1 (src/params.h:19)
constexpr uint32_t kRefPrimes[3] = {16760833u, 2147352577u, 2130706433u};

void aes_sbox(uint8_t out[256]);
// FIPS-197 key expansion into 60 big-endian round-key words
void aes_key_expand(const uint8_t key[32], uint32_t w[60]);

int sampler_init_device();

// CPU stream mapping: nstreams independent AES-CTR streams (round keys d_rkeys[nstreams][60],
// nonce 0, counter 0), each running `calls` consecutive sampler calls of n samples with
// sigma index sig; residues written to d_out[nstreams][calls][3][n].
uint32_t cpu_map_refills(uint32_t calls, uint32_t n, int sig);
size_t cpu_map_workspace_bytes(uint32_t nstreams, uint32_t calls, uint32_t n, int sig);
int sample_cpu_map(int sig, uint32_t nstreams, const uint32_t *d_rkeys, uint32_t calls, uint32_t n,
                   uint32_t *d_out, void *ws, uint32_t *d_status, int num_sms, cudaStream_t s);

// The candidate form of the CPU mapping, for consumers that gather the samples themselves:
// cand[stream][refill][8] signed candidates, amask[stream][refill] accept bits and
// call_start[stream][calls+1] (refill index where each call starts; the last entry is the
// end of the last call).  Sample j of call c is the j-th accepted candidate of refills
// call_start[c] .. call_start[c+1]-1, in order.
struct CpuMapCandidates {
  const int64_t *cand;
  const uint8_t *amask;
  const uint32_t *call_start;
  uint32_t refills;  // per stream
  // per-stream exclusive prefix of accept counts: elocal[t] + tile_off[t / 4096]
  const uint32_t *elocal, *tile_off;
  uint32_t tiles;
};
int sample_cpu_map_candidates(int sig, uint32_t nstreams, const uint32_t *d_rkeys, uint32_t calls, uint32_t n,
                              void *ws, uint32_t *d_status, int num_sms, cudaStream_t s, CpuMapCandidates *out);

// GPU counter mapping: polynomials poly0 .. poly0+npolys-1 of one key, residues to
// d_out[npolys][3][n].
int sample_gpu_map(int sig, const uint32_t *d_rkey, uint32_t poly0, uint32_t npolys, uint32_t n,
                   uint32_t *d_out, uint32_t *d_status, cudaStream_t s);

// uniform a (sample_polya): d_a[3][n]
int sample_polya(const uint32_t *d_rkey, uint32_t n, uint32_t *d_a, cudaStream_t s);

}  // namespace cufe
