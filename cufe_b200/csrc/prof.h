// prof.h -- optional per-kernel timing: CUDA events recorded around each launch on the
// launching stream, summed per kernel name when collected.  Off unless enabled on a context.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

namespace cufe {

struct Prof {
  bool on = false;
  struct Rec {
    const char *name;
    cudaEvent_t a, b;
  };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  std::map<std::string, std::pair<long long, double>> acc;  // launches, ms
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  void collect() {
    for (auto &r : pending) {
      cudaEventSynchronize(r.b);
      float ms = 0;
      cudaEventElapsedTime(&ms, r.a, r.b);
      auto &v = acc[r.name];
      v.first += 1;
      v.second += ms;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
  ~Prof() {
    for (auto &r : pending) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

// the profiler of the context whose call is running on this thread (set by the C ABI)
extern thread_local Prof *t_prof;

struct ProfScope {
  Prof *p;
  cudaStream_t s;
  const char *name;
  cudaEvent_t a = nullptr;
  ProfScope(const char *nm, cudaStream_t st) : p(t_prof), s(st), name(nm) {
    if (p && p->on) {
      a = p->get();
      cudaEventRecord(a, s);
    }
  }
  ~ProfScope() {
    if (p && p->on) {
      cudaEvent_t b = p->get();
      cudaEventRecord(b, s);
      p->pending.push_back({name, a, b});
    }
  }
};

}  // namespace cufe
