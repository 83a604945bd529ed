// counters.hpp — launch counting and per-kernel-family CUDA-event timing.
//
// Every kernel launch in this library goes through SG_LAUNCH_SCOPE(name, stream):
// it bumps the launch counter and, while profiling is enabled, brackets the
// launch with an event pair recorded on the launching stream. The event pairs
// are resolved (elapsed time summed per kernel family) when read.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

namespace sg {

extern std::atomic<uint64_t> g_kernel_launches;
inline void count_launches(uint64_t k) { g_kernel_launches.fetch_add(k, std::memory_order_relaxed); }

struct ProfStat {
  std::string name;
  uint64_t launches = 0;
  double total_ms = 0;
};

class Profiler {
 public:
  static Profiler& get();
  bool on() const { return on_.load(std::memory_order_relaxed); }
  void enable(bool v);
  // returns a slot id (or -1 when off); end() records the closing event
  int begin(const char* name, cudaStream_t s);
  void end(int slot, cudaStream_t s);
  std::vector<ProfStat> read();  // waits for pending events
  void reset();

 private:
  struct Pending {
    std::string name;
    cudaEvent_t a, b;
  };
  cudaEvent_t take();
  std::atomic<bool> on_{false};
  std::mutex mu_;
  std::vector<Pending> pending_;
  std::vector<cudaEvent_t> free_;
  std::vector<ProfStat> stats_;
};

struct LaunchScope {
  int slot;
  cudaStream_t s;
  LaunchScope(const char* name, cudaStream_t st) : slot(-1), s(st) {
    count_launches(1);
    if (Profiler::get().on()) slot = Profiler::get().begin(name, st);
  }
  ~LaunchScope() {
    if (slot >= 0) Profiler::get().end(slot, s);
  }
};

#define SG_CAT2(a, b) a##b
#define SG_CAT(a, b) SG_CAT2(a, b)
#define SG_LAUNCH_SCOPE(name, stream) ::sg::LaunchScope SG_CAT(_sg_scope_, __LINE__)(name, stream)

}  // namespace sg
