// Count of the kernels this library has launched (the evidence that the
// native path ran): every launch site adds one; a replayed CUDA graph adds
// its kernel nodes.
#pragma once
#include <atomic>

namespace slim {
extern std::atomic<unsigned long long> g_kernel_launches;
inline void count_launch(unsigned long long n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace slim
