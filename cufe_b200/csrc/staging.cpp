// staging.cpp -- see staging.h.
#include "staging.h"

#include <unistd.h>

#include <algorithm>
#include <cstring>

namespace cufe {

CopyPool::CopyPool(int nthreads) : n_(std::max(1, nthreads)), pid_((long)getpid()) {
  for (int i = 1; i < n_; ++i) th_.emplace_back(&CopyPool::worker, this, i);
}

CopyPool::~CopyPool() {
  if ((long)getpid() != pid_) {  // a fork()ed child: the workers live in the parent only, so
    new std::vector<std::thread>(std::move(th_));  // their handles are left alone (leaked)
    return;
  }
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  for (auto &t : th_) t.join();
}

// slice id of a copy: 64-byte aligned parts
void CopyPool::slice(int id, char *dst, const char *src, size_t bytes) const {
  const size_t part = ((bytes + n_ - 1) / n_ + 63) & ~(size_t)63;
  const size_t off = (size_t)id * part;
  if (off >= bytes) return;
  std::memcpy(dst + off, src + off, std::min(part, bytes - off));
}

void CopyPool::worker(int id) {
  uint64_t seen = 0;
  for (;;) {
    char *dst;
    const char *src;
    size_t bytes;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
      dst = dst_;
      src = src_;
      bytes = bytes_;
    }
    slice(id, dst, src, bytes);
    std::lock_guard<std::mutex> lk(mu_);
    if (--pending_ == 0) done_cv_.notify_one();
  }
}

void CopyPool::copy(void *dst, const void *src, size_t bytes) {
  if (n_ == 1 || bytes < ((size_t)1 << 20) || (long)getpid() != pid_) {
    std::memcpy(dst, src, bytes);
    return;
  }
  {
    std::lock_guard<std::mutex> lk(mu_);
    dst_ = static_cast<char *>(dst);
    src_ = static_cast<const char *>(src);
    bytes_ = bytes;
    pending_ = n_ - 1;
    ++gen_;
  }
  cv_.notify_all();
  slice(0, static_cast<char *>(dst), static_cast<const char *>(src), bytes);
  std::unique_lock<std::mutex> lk(mu_);
  done_cv_.wait(lk, [&] { return pending_ == 0; });
}

Staging::~Staging() {
  delete pool_;
  for (int i = 0; i < 2; ++i) {
    if (pin_[i]) cudaFreeHost(pin_[i]);
    if (ev_[i]) cudaEventDestroy(ev_[i]);
  }
}

bool Staging::ready() {
  if (pool_) return true;
  if (failed_) return false;
  for (int i = 0; i < 2; ++i) {
    if (cudaHostAlloc(&pin_[i], kChunk, cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      failed_ = true;
      return false;
    }
  }
  const unsigned hw = std::thread::hardware_concurrency();
  pool_ = new CopyPool((int)std::min(8u, std::max(1u, hw / 2)));
  return true;
}

cudaError_t Staging::h2d(void *dst_dev, const void *src, size_t bytes, cudaStream_t s) {
  if (bytes < kChunk || !ready()) return cudaMemcpy(dst_dev, src, bytes, cudaMemcpyHostToDevice);
  bool used[2] = {false, false};
  cudaError_t e = cudaSuccess;
  for (size_t off = 0, k = 0; off < bytes && e == cudaSuccess; off += kChunk, ++k) {
    const int slot = (int)(k & 1);
    const size_t len = std::min(kChunk, bytes - off);
    if (used[slot] && (e = cudaEventSynchronize(ev_[slot])) != cudaSuccess) break;  // its last DMA is done
    pool_->copy(pin_[slot], static_cast<const char *>(src) + off, len);
    e = cudaMemcpyAsync(static_cast<char *>(dst_dev) + off, pin_[slot], len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev_[slot], s);
    used[slot] = true;
  }
  const cudaError_t e2 = cudaStreamSynchronize(s);
  return e != cudaSuccess ? e : e2;
}

cudaError_t Staging::d2h(void *dst, const void *src_dev, size_t bytes, cudaStream_t s) {
  if (bytes < kChunk || !ready()) return cudaMemcpy(dst, src_dev, bytes, cudaMemcpyDeviceToHost);
  const size_t nchunks = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t k) {
    const size_t off = k * kChunk;
    cudaError_t e = cudaMemcpyAsync(pin_[k & 1], static_cast<const char *>(src_dev) + off,
                                    std::min(kChunk, bytes - off), cudaMemcpyDeviceToHost, s);
    return e == cudaSuccess ? cudaEventRecord(ev_[k & 1], s) : e;
  };
  cudaError_t e = issue(0);
  for (size_t k = 0; k < nchunks && e == cudaSuccess; ++k) {
    // chunk k + 1 goes into the other slot, whose host copy (chunk k - 1) has finished
    if (k + 1 < nchunks && (e = issue(k + 1)) != cudaSuccess) break;
    if ((e = cudaEventSynchronize(ev_[k & 1])) != cudaSuccess) break;
    const size_t off = k * kChunk;
    pool_->copy(static_cast<char *>(dst) + off, pin_[k & 1], std::min(kChunk, bytes - off));
  }
  const cudaError_t e2 = cudaStreamSynchronize(s);
  return e != cudaSuccess ? e : e2;
}

}  // namespace cufe
