// ORACLE TEST INFRASTRUCTURE — seeded inputs shared by the CPU oracle and the harnesses.
//
// A counter-based generator: u(seed, i) = top 53 bits of splitmix64(splitmix64(seed) ^ i)
// scaled to [0, 1). The same arithmetic is restated in markovkit_b200/inputs.py, so the CPU and
// GPU sides draw identical uniforms without sharing state. Uniform right-hand sides are
// u / sum(u); Dirichlet(1) right-hand sides are -log(1 - u) / sum(-log(1 - u)).
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace oracle {

inline std::uint64_t splitmix64(std::uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30U)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27U)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31U);
}

inline double uniform01(std::uint64_t seed, std::uint64_t i) {
    const std::uint64_t bits = splitmix64(splitmix64(seed) ^ i) >> 11U;
    return static_cast<double>(bits) * 0x1.0p-53;
}

inline std::vector<double> uniform_vector(std::uint64_t seed, std::size_t n) {
    std::vector<double> v(n);
    for (std::size_t i = 0; i < n; ++i) {
        v[i] = uniform01(seed, i);
    }
    return v;
}

inline std::vector<double> uniform_rhs(std::uint64_t seed, std::size_t n) {
    auto v = uniform_vector(seed, n);
    double total = 0.0;
    for (double x : v) {
        total += x;
    }
    for (double &x : v) {
        x /= total;
    }
    return v;
}

inline std::vector<double> dirichlet_rhs(std::uint64_t seed, std::size_t n) {
    std::vector<double> v(n);
    double total = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        v[i] = -std::log1p(-uniform01(seed, i));
        total += v[i];
    }
    for (double &x : v) {
        x /= total;
    }
    return v;
}

} // namespace oracle
