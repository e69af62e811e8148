// hg_prof.cuh -- optional per-phase timing with CUDA events on the launching
// stream, and a count of kernel launches.  Off by default; enabled with
// hg_profile_enable().  Events are recorded stream-ordered, so turning it on
// adds no host synchronisation to the launches.
#pragma once
#include <atomic>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

namespace hg {

struct PhaseRec {
  const char* name;
  cudaEvent_t a, b;
};

struct Profiler {
  std::mutex mu;
  bool on = false;
  std::vector<PhaseRec> recs;   // recorded since the last read
  std::vector<cudaEvent_t> pool;
  std::atomic<unsigned long long> launches{0};

  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};

inline Profiler& profiler() {
  static Profiler p;
  return p;
}

inline void count_launch(unsigned k = 1) { profiler().launches.fetch_add(k, std::memory_order_relaxed); }

// RAII phase marker: records an event at construction and at destruction.
class Phase {
 public:
  Phase(cudaStream_t s, const char* name) : s_(s) {
    Profiler& p = profiler();
    if (!p.on) return;
    std::lock_guard<std::mutex> g(p.mu);
    rec_.name = name;
    rec_.a = p.take();
    rec_.b = p.take();
    cudaEventRecord(rec_.a, s_);
    active_ = true;
  }
  ~Phase() {
    if (!active_) return;
    Profiler& p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    cudaEventRecord(rec_.b, s_);
    p.recs.push_back(rec_);
  }
  Phase(const Phase&) = delete;
  Phase& operator=(const Phase&) = delete;

 private:
  cudaStream_t s_;
  PhaseRec rec_{};
  bool active_ = false;
};

}  // namespace hg
