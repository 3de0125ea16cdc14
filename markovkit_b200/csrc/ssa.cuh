// Batched stochastic simulation of a reaction network (markovkit/ssa.hpp:42-113): Gillespie's
// direct method and Poisson tau-leaping, one path per thread.
//
// The network is the one of the FSP instances: S <= 4 species, R <= 16 reactions with change
// vectors, and propensities tabulated by the caller over a box 0 <= x_s <= bounds[s] (species 0
// most significant), because the device cannot call host lambdas. A path whose next state would
// leave the box stops with status kEOverflow (the caller widens the box and runs again: paths
// are a function of (seed, path index) alone, so they replay exactly).
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC 2011) keyed by the seed, with the path index and a per-path draw counter as
// the counter; each draw gives one double in [0, 1) from 53 bits. An exponential waiting time
// is -log(1 - u) / total; a reaction is chosen by the first cumulative rate above u * total
// (rates summed in reaction order, as the reference's categorical draw over its transition
// list); a Poisson count by multiplication of uniforms below mean 30 (Knuth, TAOCP vol. 2,
// 3.4.1) and by Hormann's transformed rejection PTRS above ("The transformed rejection method
// for generating Poisson random variables", 1993).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mkb {

constexpr int kSsaMaxSpecies = 4;
constexpr int kSsaMaxReactions = 16;
constexpr std::int64_t kSsaStepCap = std::int64_t(1) << 32; // jumps or leaps per path, at most

struct SsaParams {
    int S = 0, R = 0;
    int bounds[kSsaMaxSpecies] = {};
    int stride[kSsaMaxSpecies] = {}; // box index = sum_s x_s * stride[s]
    int change[kSsaMaxReactions][kSsaMaxSpecies] = {};
    int initial[kSsaMaxSpecies] = {};
    const double *rates = nullptr; // R x box_size
    std::int64_t box_size = 0;
    double final_time = 0.0;
    int method = 0;                // 0 Gillespie, 1 tau-leaping
    std::int64_t max_jumps = 0;    // Gillespie: jumps per path (capped at kSsaStepCap)
    double leap_step = 0.0, leap_epsilon = 0.03, leap_min_step = 1e-6;
    std::int64_t paths = 0;
    std::uint64_t seed = 0;
    int n_obs = 0;
    const double *obs_times = nullptr; // sorted
    int record = 0;                    // trajectory entries kept per path (0: none)
    // outputs (device)
    int *final_state = nullptr;   // paths x S
    int *observed = nullptr;      // paths x n_obs x S (n_obs > 0)
    std::int64_t *jumps = nullptr; // paths: jumps (Gillespie) or leaps (tau-leaping)
    int *status = nullptr;        // paths
    double *rec_times = nullptr;  // paths x record
    int *rec_states = nullptr;    // paths x record x S
    int *rec_count = nullptr;     // paths: entries of the full trajectory (may exceed record)
};

cudaError_t launch_ssa(const SsaParams &p, cudaStream_t stream);

} // namespace mkb
