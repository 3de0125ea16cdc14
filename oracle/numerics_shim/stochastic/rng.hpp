// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// A seeded uniform random bit generator (markovkit/ssa.hpp:42 requires the std concept).
#pragma once

#include <cstdint>
#include <random>

namespace num {

class rng {
  public:
    using result_type = std::uint64_t;
    explicit rng(std::uint64_t seed = 0) : engine_(seed) {}
    static constexpr result_type min() { return std::mt19937_64::min(); }
    static constexpr result_type max() { return std::mt19937_64::max(); }
    result_type operator()() { return engine_(); }
    double uniform() { return std::uniform_real_distribution<double>(0.0, 1.0)(engine_); }

  private:
    std::mt19937_64 engine_;
};

} // namespace num
