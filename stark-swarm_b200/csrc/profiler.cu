// profiler.cu — per-kernel-family CUDA-event timing (see counters.hpp).
#include <map>

#include "counters.hpp"

namespace sg {

std::atomic<uint64_t> g_kernel_launches{0};

Profiler& Profiler::get() {
  static Profiler p;
  return p;
}

void Profiler::enable(bool v) { on_.store(v); }

cudaEvent_t Profiler::take() {
  if (!free_.empty()) {
    cudaEvent_t e = free_.back();
    free_.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

int Profiler::begin(const char* name, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  Pending p{name, take(), take()};
  if (!p.a || !p.b) return -1;
  cudaEventRecord(p.a, s);
  pending_.push_back(p);
  return (int)pending_.size() - 1;
}

void Profiler::end(int slot, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (slot >= 0 && slot < (int)pending_.size()) cudaEventRecord(pending_[slot].b, s);
}

std::vector<ProfStat> Profiler::read() {
  std::lock_guard<std::mutex> g(mu_);
  std::map<std::string, size_t> idx;
  for (size_t i = 0; i < stats_.size(); ++i) idx[stats_[i].name] = i;
  for (auto& p : pending_) {
    float ms = 0;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      auto it = idx.find(p.name);
      if (it == idx.end()) {
        idx[p.name] = stats_.size();
        stats_.push_back(ProfStat{p.name, 0, 0});
        it = idx.find(p.name);
      }
      stats_[it->second].launches += 1;
      stats_[it->second].total_ms += ms;
    }
    free_.push_back(p.a);
    free_.push_back(p.b);
  }
  pending_.clear();
  return stats_;
}

void Profiler::reset() {
  read();
  std::lock_guard<std::mutex> g(mu_);
  stats_.clear();
}

}  // namespace sg
