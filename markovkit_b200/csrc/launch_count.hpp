// A process-wide count of this library's kernel launches (a graph launch counts its kernel
// nodes), read through mk_kernel_launches.
#pragma once

#include <atomic>
#include <cstdint>

namespace mkb {

inline std::atomic<std::uint64_t> g_kernel_launches{0};

inline void count_launches(std::uint64_t n) {
    g_kernel_launches.fetch_add(n, std::memory_order_relaxed);
}

} // namespace mkb
