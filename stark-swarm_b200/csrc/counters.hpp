// counters.hpp — process-wide count of kernels launched by this library.
#pragma once
#include <atomic>
#include <cstdint>

namespace sg {
extern std::atomic<uint64_t> g_kernel_launches;
inline void count_launches(uint64_t k) { g_kernel_launches.fetch_add(k, std::memory_order_relaxed); }
}  // namespace sg
