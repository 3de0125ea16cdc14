// Batched Krylov finite state projection on sm_100a: many solve_krylov_fsp runs
// (markovkit/fsp.hpp:190-254) in one persistent kernel, one block per instance.
#pragma once

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
    int pad = 0;
};

struct FspBatchView {
    const FspInstance *inst = nullptr;
    int n = 0;
    const double *rates = nullptr;
    double *out = nullptr;          // final distributions, box order
    FspOutcome *outcome = nullptr;
    int *queue = nullptr;           // next instance to take (atomic)
    // per-block workspace of `cap` states: Krylov basis and vectors, slot maps
    double *work = nullptr;
    int *iwork = nullptr;
    std::int64_t cap = 0;
};

// block shapes the kernel is built for (threads per block); the autotuner picks one of these
// and the number of blocks
constexpr int kFspShapes[] = {128, 256, 512};

// doubles and ints of per-block workspace for a capacity of `cap` states: the Krylov basis
// (krylov_dim + 1 vectors) and five more vectors; the box-to-slot map, the slot list, a
// compaction buffer and the first-discoverer map of the expansion
__host__ __device__ inline std::int64_t fsp_work_doubles(std::int64_t cap) {
    return (kFspMaxKrylov + 6) * cap;
}
__host__ __device__ inline std::int64_t fsp_work_ints(std::int64_t cap) { return 4 * cap; }
std::size_t fsp_shared_bytes();

// resident blocks per SM of the kernel with `threads` threads per block
int fsp_blocks_per_sm(int threads);

// instances are taken in queue order: v.inst[0], v.inst[1], ...; *v.queue must be 0
cudaError_t launch_fsp_batch(const FspBatchView &v, int threads, int blocks,
                             cudaStream_t stream);

} // namespace mkb
