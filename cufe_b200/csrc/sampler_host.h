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
// device key expansion: d_rk[i][60] = aes_key_expand(d_seeds[d_perm ? d_perm[i] : i])
int expand_keys_device(const uint8_t *d_seeds, const uint32_t *d_perm, uint32_t count, uint32_t *d_rk,
                       cudaStream_t s);

// CPU stream mapping: nstreams independent AES-CTR streams (round keys d_rkeys[nstreams][60],
// nonce 0, counter 0), each running `calls` consecutive sampler calls of n samples with
// sigma index sig; residues written to d_out[nstreams][calls][3][n].
uint32_t cpu_map_refills(uint32_t calls, uint32_t n, int sig);
size_t cpu_map_workspace_bytes(uint32_t nstreams, uint32_t calls, uint32_t n, int sig);
int sample_cpu_map(int sig, uint32_t nstreams, const uint32_t *d_rkeys, uint32_t calls, uint32_t n,
                   uint32_t *d_out, void *ws, uint32_t *d_status, int num_sms, cudaStream_t s);

// Segmented form: S CPU-mapping streams of different lengths.  Stream s runs calls[s]
// sampler calls of n[s] samples; its refills occupy [roff[s], roff[s+1]) of the flattened
// refill space, its scan tiles [toff[s], toff[s+1]), its call starts
// call_start[coff[s] + s .. coff[s+1] + s] (calls + 1 entries), and the scatter writes its
// residues to out[ooff[s] + c * 3 n[s] ...][3][n[s]].  Round keys rkeys[s][60].
struct SegDev {
  uint32_t nstreams;
  const uint32_t *n, *calls, *toff;
  const uint64_t *roff, *coff, *ooff;
};
struct SegSizes {
  uint32_t nstreams;
  uint64_t refills;
  uint32_t tiles;
  uint64_t calls;
  uint32_t max_calls;  // the largest calls[s]
  bool doubling;       // call starts by pointer doubling (its tables are part of the scratch)
};
// How the call starts of the CPU mapping are found.  Pointer doubling is parallel over
// refills and calls but costs bit_length(max_calls) table passes over all refills (and as
// many words of scratch per refill); the serial walk (one warp per stream) costs a dependent
// search per call.  Doubling is chosen when it is estimated cheaper and stays below 32 Mi
// refills; set_call_search(1) forces the walk.  The choice is fixed in SegSizes when a
// scratch is sized.
void set_call_search(int mode);
int get_call_search();
bool seg_auto_doubling(uint64_t refills, uint32_t max_calls);
struct SegLayout {
  size_t n, calls, toff, roff, coff, ooff, bytes;
};
// the tables of S streams in one buffer (device or host, same layout)
SegLayout seg_layout(uint32_t S);
SegDev seg_bind(void *base, uint32_t S);
// host: fill the tables (refills per stream from cpu_map_refills) into a host buffer of
// seg_layout(S).bytes; ooff may be NULL (candidates only)
SegSizes seg_fill_host(int sig, uint32_t S, const uint32_t *calls, const uint32_t *n, const uint64_t *ooff,
                       void *host_base);
size_t seg_scratch_bytes(const SegSizes &z);

// segmented run: candidates, scan, call starts and the scatter of the residues to d_out
int sample_cpu_map_seg(int sig, const SegDev &sg, const SegSizes &z, const uint32_t *d_rkeys, uint32_t *d_out,
                       void *scratch, uint32_t *d_status, int num_sms, cudaStream_t s);

// GPU counter mapping: polynomials poly0 .. poly0+npolys-1 of one key, residues to
// d_out[npolys][3][n].
int sample_gpu_map(int sig, const uint32_t *d_rkey, uint32_t poly0, uint32_t npolys, uint32_t n,
                   uint32_t *d_out, uint32_t *d_status, cudaStream_t s);

// uniform a (sample_polya): d_a[3][n]
int sample_polya(const uint32_t *d_rkey, uint32_t n, uint32_t *d_a, cudaStream_t s);

}  // namespace cufe
