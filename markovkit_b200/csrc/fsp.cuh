// Batched Krylov finite state projection on sm_100a: many solve_krylov_fsp runs
// (markovkit/fsp.hpp:190-254) in one persistent kernel, one block per instance.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mkb {

constexpr int kFspMaxSpecies = 4;
constexpr int kFspMaxReactions = 16;
constexpr int kFspMaxKrylov = 30; // krylov_dim <= 30: the augmented Hessenberg fits 32 x 32

// One instance on the device. States live in the box 0 <= x_s <= bound_s, numbered in mixed
// radix with species 0 most significant.
struct FspInstance {
    int S = 1, R = 0;
    int box = 1;                        // states in the box
    int bound[kFspMaxSpecies] = {};
    int stride[kFspMaxSpecies] = {};
    int change[kFspMaxReactions][kFspMaxSpecies] = {};
    int initial = 0;                    // box index of the initial state
    int layers = 1;
    int krylov_dim = 30;
    int index = 0;                      // position of the outcome in FspBatchView::outcome
    std::int64_t rate_offset = 0;       // rates[r * box + i] at rate_offset
    std::int64_t out_offset = 0;        // final distribution (box order) at out_offset
    std::int64_t max_steps = 0;
    double final_time = 0;
    double tolerance = 1e-6, initial_step = 1.0, step_growth = 2.0;
    double drop_probability = 1e-10, drop_derivative = 1e-16;
    double krylov_tol = 1e-8;
    // 0: solve_krylov_fsp (fsp.hpp:190-254); 1: solve_adaptive_fsp (fsp.hpp:108-188), whose steps
    // take step_scale / (expected jump rate) and prune the least likely prune_fraction of the
    // support where their flux is below flux_tolerance of the total, and any state below
    // min_probability
    int method = 0;
    int pad = 0;
    double step_scale = 1.0, prune_fraction = 0.1, flux_tolerance = 1e-6, min_probability = 0.0;
};

// per-instance outcome
struct FspOutcome {
    double time = 0;
    std::int64_t attempts = 0;
    std::int64_t accepted = 0;
    std::int64_t support = 0;
    std::int64_t substeps = 0;  // expv time steps
    std::int64_t applies = 0;   // operator applies (Arnoldi steps and the extra ones)
    int status = 0; // 0 ok, 1 expv tolerance too high, 2 step limit, 3 non-finite
    int clipped = 0; // bit s: an expansion met a jump to a state above bounds[s]
};

struct FspBatchView {
    const FspInstance *inst = nullptr;
    int n = 0;
    const double *rates = nullptr;
    double *out = nullptr;          // final distributions, box order
    FspOutcome *outcome = nullptr;
    int *queue = nullptr;           // next instance to take (atomic)
    // per-block workspace of `cap` states (see fsp_work_doubles / fsp_work_ints)
    double *work = nullptr;
    int *iwork = nullptr;
    std::int64_t cap = 0;
    int rmax = 0;                   // most reactions of any instance
    // shared memory per block beyond the fixed part, for the vectors, the assembled operator
    // and the Krylov basis of an instance small enough to keep there
    std::size_t arena_bytes = 0;
};

// block sizes the kernel is built for; the autotuner picks one and the blocks per SM
constexpr int kFspShapes[] = {128, 256, 512};

// Per-block global workspace for `cap` states and up to `rmax` reactions. Doubles: the Krylov
// basis (krylov_dim + 1 vectors), five vectors and the assembled operator (rmax coefficients
// and the exit rate per state). Ints: the box-to-slot map, the slot list, a compaction buffer,
// the first-discoverer map of the expansion and rmax neighbour slots per state.
__host__ __device__ inline std::int64_t fsp_work_doubles(std::int64_t cap, int rmax) {
    return (kFspMaxKrylov + 7 + rmax) * cap;
}
__host__ __device__ inline std::int64_t fsp_work_ints(std::int64_t cap, int rmax) {
    return (4 + rmax) * cap;
}

// the fixed shared memory of a block
std::size_t fsp_fixed_shared_bytes();

// Largest arena with which `blocks_per_sm` blocks of `threads` threads fit on one SM (0 if
// they do not fit even without one).
std::size_t fsp_arena_bytes(int threads, int blocks_per_sm);

// most resident blocks per SM of the kernel with `threads` threads and no arena
int fsp_blocks_per_sm(int threads);

// instances are taken in queue order: v.inst[0], v.inst[1], ...; *v.queue must be 0
cudaError_t launch_fsp_batch(const FspBatchView &v, int threads, int blocks,
                             cudaStream_t stream);

} // namespace mkb
