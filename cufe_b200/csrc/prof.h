// prof.h -- optional per-kernel timing: CUDA events recorded around each named launch group
// on the launching stream, summed per name with the number of kernels launched inside it.
// Off unless enabled on a context.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

namespace cufe {

struct Prof {
  bool on = false;
  long long kernels = 0;  // kernel launches while on (all of them, inside a scope or not)
  struct Rec {
    const char *name;
    cudaEvent_t a, b;
    long long kernels;  // launched inside the scope
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
      v.first += r.kernels;
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
// kernel launches issued by this thread; every launch site is written `note_launch(), k<<<...>>>`
extern thread_local long long t_launches;
inline void note_launch() {
  ++t_launches;
  if (t_prof && t_prof->on) ++t_prof->kernels;
}

struct ProfScope {
  Prof *p;
  cudaStream_t s;
  const char *name;
  cudaEvent_t a = nullptr;
  long long k0 = t_launches;
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
      p->pending.push_back({name, a, b, t_launches - k0});
    }
  }
};

}  // namespace cufe
