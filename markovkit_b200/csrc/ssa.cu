// Batched Gillespie and tau-leaping paths (ssa.cuh).
#include "host_model.hpp"
#include "launch_count.hpp"
#include "ssa.cuh"

#include <cmath>

namespace mkb {
namespace {

constexpr int kSsaThreads = 128;
constexpr int kPoissonTries = 1000; // rejection loops end here (acceptance is ~0.9 per try)

// Philox4x32-10: ten rounds of two 32x32 -> 64-bit products with the published multipliers and
// Weyl key increments
struct Philox {
    std::uint32_t k0, k1;
    std::uint32_t c[4];
    double spare = 0.0;
    bool has_spare = false;

    __device__ Philox(std::uint64_t seed, std::uint64_t path)
        : k0(static_cast<std::uint32_t>(seed)), k1(static_cast<std::uint32_t>(seed >> 32)),
          c{0U, 0U, static_cast<std::uint32_t>(path), static_cast<std::uint32_t>(path >> 32)} {}

    __device__ void block(std::uint32_t (&out)[4]) const {
        std::uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
        std::uint32_t a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            const std::uint64_t p0 = static_cast<std::uint64_t>(0xD2511F53U) * x0;
            const std::uint64_t p1 = static_cast<std::uint64_t>(0xCD9E8D57U) * x2;
            const std::uint32_t hi0 = static_cast<std::uint32_t>(p0 >> 32), lo0 = static_cast<std::uint32_t>(p0);
            const std::uint32_t hi1 = static_cast<std::uint32_t>(p1 >> 32), lo1 = static_cast<std::uint32_t>(p1);
            x0 = hi1 ^ x1 ^ a;
            x1 = lo1;
            x2 = hi0 ^ x3 ^ b;
            x3 = lo0;
            a += 0x9E3779B9U;
            b += 0xBB67AE85U;
        }
        out[0] = x0;
        out[1] = x1;
        out[2] = x2;
        out[3] = x3;
    }

    // a double in [0, 1): 53 bits of one 64-bit half of a block; two per block
    __device__ double uniform() {
        if (has_spare) {
            has_spare = false;
            return spare;
        }
        std::uint32_t o[4];
        block(o);
        if (++c[0] == 0U) {
            ++c[1];
        }
        const double scale = 1.0 / 9007199254740992.0; // 2^-53
        const std::uint64_t m0 = ((static_cast<std::uint64_t>(o[0]) << 32) | o[1]) >> 11;
        const std::uint64_t m1 = ((static_cast<std::uint64_t>(o[2]) << 32) | o[3]) >> 11;
        spare = static_cast<double>(m1) * scale;
        has_spare = true;
        return static_cast<double>(m0) * scale;
    }
};

// Poisson(mu): products of uniforms below 30, PTRS above; the loops are bounded
__device__ std::int64_t poisson(Philox &rng, double mu) {
    if (!(mu > 0.0)) {
        return 0;
    }
    if (mu < 30.0) {
        const double limit = exp(-mu);
        double prod = 1.0;
        std::int64_t k = 0;
        do {
            ++k;
            prod *= rng.uniform();
        } while (prod > limit && k < 4 * kPoissonTries);
        return k - 1;
    }
    const double smu = sqrt(mu);
    const double b = 0.931 + 2.53 * smu;
    const double a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    const double log_mu = log(mu);
    for (int tries = 0; tries < kPoissonTries; ++tries) {
        const double u = rng.uniform() - 0.5;
        const double v = rng.uniform();
        const double us = 0.5 - fabs(u);
        const double k = floor((2.0 * a / us + b) * u + mu + 0.43);
        if (us >= 0.07 && v <= vr) {
            return static_cast<std::int64_t>(k);
        }
        if (k < 0.0 || (us < 0.013 && v > us)) {
            continue;
        }
        if (log(v) + log(inv_alpha) - log(a / (us * us) + b) <= -mu + k * log_mu - lgamma(k + 1.0)) {
            return static_cast<std::int64_t>(k);
        }
    }
    return static_cast<std::int64_t>(floor(mu));
}

// the propensities of the listed transitions of x (reaction_network::transitions: a reaction is
// listed when its result has no negative count and its rate is > 0), 0 for the others
template <int NR>
__device__ double propensities(const SsaParams &p, const int (&x)[kSsaMaxSpecies], double (&a)[NR]) {
    std::int64_t idx = 0;
#pragma unroll
    for (int s = 0; s < kSsaMaxSpecies; ++s) {
        if (s < p.S) {
            idx += static_cast<std::int64_t>(x[s]) * p.stride[s];
        }
    }
    double total = 0.0;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        a[r] = 0.0;
        if (r >= p.R) {
            continue;
        }
        bool valid = true;
#pragma unroll
        for (int s = 0; s < kSsaMaxSpecies; ++s) {
            valid = valid && (s >= p.S || x[s] + p.change[r][s] >= 0);
        }
        const double rate = __ldg(p.rates + static_cast<std::int64_t>(r) * p.box_size + idx);
        if (valid && rate > 0.0) {
            a[r] = rate;
            total += rate;
        }
    }
    return total;
}

__device__ void write_state(int *dst, const int (&x)[kSsaMaxSpecies], int S) {
    for (int s = 0; s < S; ++s) {
        dst[s] = x[s];
    }
}

// NR: the reactions' count rounded up to 4, 8 or 16 (the propensities stay in registers)
template <int NR>
__global__ void __launch_bounds__(kSsaThreads) ssa_kernel(const SsaParams p) {
    const std::int64_t path = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
    if (path >= p.paths) {
        return;
    }
    const int S = p.S;
    Philox rng(p.seed, static_cast<std::uint64_t>(path));
    int x[kSsaMaxSpecies] = {};
    for (int s = 0; s < S; ++s) {
        x[s] = p.initial[s];
    }
    int *obs_out = p.n_obs > 0 ? p.observed + path * p.n_obs * S : nullptr;
    int k_obs = 0;
    std::int64_t entries = 0;
    auto record = [&](double t) {
        if (entries < p.record) {
            p.rec_times[path * p.record + entries] = t;
            write_state(p.rec_states + (path * p.record + entries) * S, x, S);
        }
        ++entries;
    };
    auto observe_before = [&](double t) {
        while (k_obs < p.n_obs && p.obs_times[k_obs] < t) {
            write_state(obs_out + k_obs * S, x, S);
            ++k_obs;
        }
    };
    record(0.0);
    double a[NR];
    double t = 0.0;
    std::int64_t steps = 0;
    int status = kOk;
    if (p.method == 0) {
        // gillespie (ssa.hpp:42-74)
        const std::int64_t cap = p.max_jumps < kSsaStepCap ? p.max_jumps : kSsaStepCap;
        for (;;) {
            if (steps >= cap) {
                status = p.max_jumps > cap ? kENotConv : kOk;
                break;
            }
            const double total = propensities<NR>(p, x, a);
            if (!(total > 0.0)) {
                break;
            }
            t += -log(1.0 - rng.uniform()) / total;
            if (t > p.final_time) {
                break;
            }
            const double target = rng.uniform() * total;
            double acc = 0.0;
            int chosen = -1;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                if (a[r] > 0.0) {
                    acc += a[r];
                    if (chosen < 0 && target < acc) {
                        chosen = r;
                    }
                }
            }
            if (chosen < 0) { // rounding at the top end: the last listed transition
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    chosen = a[r] > 0.0 ? r : chosen;
                }
            }
            int y[kSsaMaxSpecies] = {};
            bool inside = true;
            for (int s = 0; s < S; ++s) {
                y[s] = x[s] + p.change[chosen][s];
                inside = inside && y[s] <= p.bounds[s];
            }
            if (!inside) {
                status = kEOverflow;
                break;
            }
            observe_before(t);
            for (int s = 0; s < S; ++s) {
                x[s] = y[s];
            }
            ++steps;
            record(t);
        }
        // a path that stopped short of max_jumps holds its last state until final_time
        if (status == kOk && steps < p.max_jumps) {
            record(p.final_time);
        }
    } else {
        // tau_leaping (ssa.hpp:83-111)
        while (t < p.final_time) {
            if (steps >= kSsaStepCap) {
                status = kENotConv;
                break;
            }
            const double total = propensities<NR>(p, x, a);
            if (!(total > 0.0)) {
                break;
            }
            double dt = p.leap_step > 0.0 ? p.leap_step : fmax(p.leap_min_step, p.leap_epsilon / total);
            dt = fmin(dt, p.final_time - t);
            t += dt;
            std::int64_t next[kSsaMaxSpecies] = {};
            for (int s = 0; s < S; ++s) {
                next[s] = x[s];
            }
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                if (!(a[r] > 0.0)) {
                    continue;
                }
                const std::int64_t fired = poisson(rng, a[r] * dt);
                for (int s = 0; s < S; ++s) {
                    const std::int64_t v = next[s] + fired * p.change[r][s];
                    next[s] = v > 0 ? v : 0;
                }
            }
            bool inside = true;
            for (int s = 0; s < S; ++s) {
                inside = inside && next[s] <= p.bounds[s];
            }
            if (!inside) {
                status = kEOverflow;
                break;
            }
            observe_before(t);
            for (int s = 0; s < S; ++s) {
                x[s] = static_cast<int>(next[s]);
            }
            ++steps;
            record(t);
        }
    }
    // observations after the last change hold the last state
    while (k_obs < p.n_obs) {
        write_state(obs_out + k_obs * S, x, S);
        ++k_obs;
    }
    write_state(p.final_state + path * S, x, S);
    p.jumps[path] = steps;
    p.status[path] = status;
    if (p.rec_count) {
        p.rec_count[path] = static_cast<int>(entries < (std::int64_t(1) << 30) ? entries : (std::int64_t(1) << 30));
    }
}

} // namespace

cudaError_t launch_ssa(const SsaParams &p, cudaStream_t stream) {
    if (p.paths <= 0) {
        return cudaSuccess;
    }
    const std::int64_t blocks = (p.paths + kSsaThreads - 1) / kSsaThreads;
    if (blocks > 0x7fffffffLL) {
        return cudaErrorInvalidValue;
    }
    count_launches(1);
    const auto grid = static_cast<unsigned>(blocks);
    if (p.R <= 4) {
        ssa_kernel<4><<<grid, kSsaThreads, 0, stream>>>(p);
    } else if (p.R <= 8) {
        ssa_kernel<8><<<grid, kSsaThreads, 0, stream>>>(p);
    } else {
        ssa_kernel<kSsaMaxReactions><<<grid, kSsaThreads, 0, stream>>>(p);
    }
    return cudaGetLastError();
}

} // namespace mkb
