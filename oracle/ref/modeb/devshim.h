/*
 * devshim.h -- lets the reference's GPU sampler code (cuFE src/sample_gpu.cu kernel bodies,
 * src/AES.cuh, src/sampler.cuh, src/arith_rns.cuh, src/params_gpu.cuh, src/consts.cuh) compile
 * and run unmodified as host C++, one CUDA block at a time.  TEST INFRASTRUCTURE ONLY: the
 * result pins the oracle's restatement of the GPU counter-to-sample mapping; nothing here is
 * part of the product.
 *
 *  - CUDA qualifiers: __global__/__device__/__host__/__constant__ vanish, __shared__ becomes a
 *    function-local static (one block runs at a time, so one copy is what a block sees).
 *  - threadIdx / blockIdx are globals the block scheduler sets before it resumes a thread.
 *  - __syncthreads() yields to the scheduler (modeb_host.cpp): every live thread runs to its
 *    next barrier (or to its end) before any thread continues, which is what the barrier in
 *    the AES table loader (src/AES.cuh:399) needs: all 256 table columns stored before the
 *    first lookup.  Threads reach that barrier a different number of times (one per refill);
 *    the table contents never change after the first load, so the extra generations do not
 *    change any output.
 *  - __byte_perm(x, y, s): PTX prmt in its default mode, as the CUDA documentation defines it
 *    (byte n of the result is byte s[4n+2:4n] of the eight bytes {y, x}).
 *  - int64_t becomes dev_i64, a 64-bit integer with the device's semantics where host and
 *    device differ on this code: a double -> int64 conversion saturates (cvt.rzi.s64.f64;
 *    NaN gives 0) where x86 gives INT64_MIN, and `v << e` is 0 unless 0 <= e <= 63 where x86
 *    masks e to 6 bits.  Both were measured on a B200 with nvcc's default flags (rounding
 *    probe: saturated conversions, zero for every shift count in [-2048, 2047] outside
 *    [0, 63]).  Signed overflow wraps (-fwrapv), as device integer arithmetic does.
 *  - Floating point: the same probe found that nvcc does not fuse `vx - floor(vx)` when vx is
 *    a product with another use; the Horner steps are single-use products that both nvcc and
 *    GCC (-ffp-contract=fast, FMA available) fuse.  So the host build rounds as the device.
 */
#ifndef CUFE_MODEB_DEVSHIM_H
#define CUFE_MODEB_DEVSHIM_H

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <type_traits>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static
#define __forceinline__ inline

struct cufe_dim3 {
  unsigned int x, y, z;
};
extern cufe_dim3 threadIdx, blockIdx, blockDim, gridDim;

void __syncthreads(void);

static inline uint32_t __byte_perm(uint32_t x, uint32_t y, uint32_t s) {
  const uint64_t b = ((uint64_t)y << 32) | x;
  uint32_t r = 0;
  for (int n = 0; n < 4; ++n) r |= (uint32_t)((b >> (8 * ((s >> (4 * n)) & 7))) & 0xff) << (8 * n);
  return r;
}

struct dev_i64 {
  long v;
  dev_i64() = default;
  template <class T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
  dev_i64(T x) : v((long)x) {}
  dev_i64(double d) {
    if (d != d) v = 0;
    else if (d >= 9223372036854775808.0) v = 0x7fffffffffffffffL;
    else if (d < -9223372036854775808.0) v = (long)(-0x7fffffffffffffffL - 1);
    else v = (long)d;
  }
  operator long() const { return v; }
  template <class T> dev_i64 &operator+=(T o) { v = (long)((unsigned long)v + (unsigned long)(long)o); return *this; }
  template <class T> dev_i64 &operator-=(T o) { v = (long)((unsigned long)v - (unsigned long)(long)o); return *this; }
  template <class T> dev_i64 &operator&=(T o) { v &= (long)o; return *this; }
  template <class T> dev_i64 &operator|=(T o) { v |= (long)o; return *this; }
  template <class T> dev_i64 &operator^=(T o) { v ^= (long)o; return *this; }
  template <class T> dev_i64 &operator<<=(T e) { *this = (long)v << dev_i64(e); return *this; }
  template <class T> dev_i64 &operator>>=(T e) { v >>= (long)e; return *this; }
};
static_assert(sizeof(dev_i64) == 8, "dev_i64 must overlay an int64");

/* integer << dev_i64: the device shift, 0 unless 0 <= e <= 63 */
template <class T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
static inline T operator<<(T x, const dev_i64 &e) {
  return (e.v >= 0 && e.v <= 63) ? (T)((unsigned long long)x << e.v) : (T)0;
}

/* from here on, the reference's int64_t is the device-semantics integer */
#define int64_t dev_i64

#endif
