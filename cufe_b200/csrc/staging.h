// staging.h -- host <-> device copies of caller-owned pageable buffers through pinned slots.
//
// cudaMemcpy from pageable memory stages through a driver buffer with one host thread.  Here
// a small pool of host threads moves each chunk between the caller's buffer and one of two
// pinned slots while the copy engine moves the previous chunk, so the host copy and the DMA
// overlap and the host side runs at several threads' memory bandwidth.  Synchronous, like
// cudaMemcpy: the call returns when the data has arrived.
#pragma once
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <thread>
#include <vector>

namespace cufe {

// memcpy split over n host threads (the caller takes the first slice)
class CopyPool {
 public:
  explicit CopyPool(int nthreads);
  ~CopyPool();
  CopyPool(const CopyPool &) = delete;
  CopyPool &operator=(const CopyPool &) = delete;
  void copy(void *dst, const void *src, size_t bytes);
  int threads() const { return n_; }

 private:
  void worker(int id);
  void slice(int id, char *dst, const char *src, size_t bytes) const;
  int n_;
  long pid_;  // the process whose threads these are (a fork()ed child copies alone)
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t bytes_ = 0;
  uint64_t gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

class Staging {
 public:
  static constexpr size_t kChunk = (size_t)8 << 20;
  Staging() = default;
  ~Staging();
  Staging(const Staging &) = delete;
  Staging &operator=(const Staging &) = delete;
  // below kChunk, or when the pinned slots cannot be had, a plain cudaMemcpy
  cudaError_t h2d(void *dst_dev, const void *src, size_t bytes, cudaStream_t s);
  cudaError_t d2h(void *dst, const void *src_dev, size_t bytes, cudaStream_t s);

 private:
  bool ready();
  CopyPool *pool_ = nullptr;
  void *pin_[2] = {nullptr, nullptr};
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  bool failed_ = false;
};

}  // namespace cufe
