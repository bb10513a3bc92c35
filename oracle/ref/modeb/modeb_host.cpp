/*
 * modeb_host.cpp -- runs the reference's GPU Gaussian sampler kernels (cuFE
 * src/sample_gpu.cu:40-99 gaussian_sampler_S1_gpu, :101-161 _S2_gpu, :217-289 _S3_gpu, with
 * src/AES.cuh:380-435 encAES256OneTblReuseRpt, :653-665 aes256ctr_squeezeblocks_gpu and
 * src/sampler.cuh) on the host, one block at a time, to pin the oracle's restatement of the GPU
 * counter-to-sample mapping (mode B) to the reference's own code.  TEST INFRASTRUCTURE ONLY.
 *
 * The kernel bodies are compiled unmodified: oracle/ref/build_ref.py copies their text out of
 * the reference tree into the build directory (oracle/_ref/modeb/, never committed) and this
 * file includes it after the reference's own headers; devshim.h supplies the CUDA keywords
 * and the device semantics (see there).  Each CUDA thread of a block is a ucontext coroutine;
 * __syncthreads() returns control to the block scheduler below.
 *
 * Reference layout at the shipped parameters (src/params.h: N = 4096; src/params_gpu.cuh:
 * THREAD = 512, LEN_THREAD = 8): block `bid` writes polynomial `bid`, thread t its
 * coefficients 8t..8t+7 of all three residues.  Only blockIdx.y = 0 is run: the S2/S3 kernels
 * read the key of instance y at a 240-word stride from a buffer packed at a 240-byte stride
 * (src/sample_gpu.cu:125 against src/rlwe_sife_gpu.cu:117), so only instance 0 is defined.  S3
 * adds its samples into a ciphertext buffer and also writes an uninitialised fourth residue
 * into the next polynomial (src/sample_gpu.cu:284); the buffer here starts at zero and has room
 * for that write, and only the block's own three residues are returned.
 */
#include "devshim.h"

#include <ucontext.h>

#include <vector>

cufe_dim3 threadIdx, blockIdx, blockDim, gridDim;

#include "params.h"
#include "AES.cuh"
#include "sampler.cuh"
#include "arith_rns.cuh"
#include "consts.cuh"

#include "sample_gpu_kernels.inc"

namespace {

constexpr size_t kStack = 128 * 1024;

ucontext_t g_sched;
std::vector<ucontext_t> g_ctx;
std::vector<char> g_done;
unsigned g_cur;
int g_sig;
uint8_t *g_rk;
uint32_t *g_out;

void thread_main() {
  switch (g_sig) {
    case 0: gaussian_sampler_S1_gpu(g_rk, g_out); break;
    case 1: gaussian_sampler_S2_gpu(g_rk, g_out); break;
    default: gaussian_sampler_S3_gpu(g_rk, g_out); break;
  }
  g_done[g_cur] = 1;
  swapcontext(&g_ctx[g_cur], &g_sched);
}

/* run every thread of block `bid` to completion, barrier generation by generation */
int run_block(unsigned bid, unsigned nthreads) {
  static std::vector<std::vector<char>> stacks;  // reused across blocks
  if (stacks.size() < nthreads) stacks.resize(nthreads, std::vector<char>(kStack));
  g_ctx.assign(nthreads, ucontext_t{});
  g_done.assign(nthreads, 0);
  blockIdx = {bid, 0, 0};
  blockDim = {nthreads, 1, 1};
  gridDim = {bid + 1, 1, 1};
  for (unsigned t = 0; t < nthreads; ++t) {
    if (getcontext(&g_ctx[t])) return -1;
    g_ctx[t].uc_stack.ss_sp = stacks[t].data();
    g_ctx[t].uc_stack.ss_size = kStack;
    g_ctx[t].uc_link = &g_sched;
    makecontext(&g_ctx[t], thread_main, 0);
  }
  for (unsigned gen = 0;; ++gen) {
    bool live = false;
    for (unsigned t = 0; t < nthreads; ++t) {
      if (g_done[t]) continue;
      live = true;
      g_cur = t;
      threadIdx = {t, 0, 0};
      if (swapcontext(&g_sched, &g_ctx[t])) return -1;
    }
    if (!live) return 0;
    if (gen > 100000) return -2;  // a block needs one generation per refill (a handful)
  }
}

}  // namespace

void __syncthreads(void) { swapcontext(&g_ctx[g_cur], &g_sched); }

extern "C" {

/* AESPrepareKey (src/AES.cuh:667-764) on a 32-byte seed: the 240-byte round-key buffer the
 * reference copies to the device (src/sample_gpu.cu:176-177) */
void modeb_prepare_key(const unsigned char seed[32], unsigned char rk[240]) {
  char buf[240];
  memset(buf, 0, sizeof buf);
  AESPrepareKey(buf, seed, 256);
  memcpy(rk, buf, 240);
}

/* one block of the sigma_{sig+1} kernel keyed by the 32-byte seed: out[3][SIFE_N] = the residues
 * of polynomial `bid` (0 <= bid < 4096).  Returns 0, or a negative value if the scheduler failed. */
int modeb_block(int sig, const unsigned char seed[32], int bid, uint32_t *out) {
  if (sig < 0 || sig > 2 || bid < 0 || bid >= 4096) return -3;
  static unsigned char rk[240];
  modeb_prepare_key(seed, rk);
  const size_t poly = (size_t)SIFE_NMODULI * SIFE_N;
  std::vector<uint32_t> buf((size_t)(bid + 2) * poly + SIFE_N, 0);
  g_sig = sig;
  g_rk = rk;
  g_out = buf.data();
  const int rc = run_block((unsigned)bid, THREAD);
  if (rc) return rc;
  memcpy(out, buf.data() + (size_t)bid * poly, poly * 4);
  return 0;
}

int modeb_n(void) { return SIFE_N; }

}  // extern "C"
