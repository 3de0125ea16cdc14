// The aggregate-block smoother of population_multigrid (markovkit/rdme/multigrid.hpp:239-341,
// relaxation::aggregate_block), and the weighted Jacobi smoothing the reference keeps on the
// sectors a level factors directly (multigrid.hpp:309-317 when a level has no blocks).
//
// A level's states are grouped once per coarse voxel a: the states that agree outside a's fine
// voxels form one block (groups of one state are skipped), each with the dense inverse of A
// restricted to it. One sweep visits the coarse voxels in order (backwards after the coarse
// correction); at each, every block of a solves A_bb e_b = r_b from the residual before any of
// a's blocks moves x, then x += e over the blocks. The residual r_b = rhs_b - (A x)_b is formed
// from the rows of A of the block's states, stored at set-up; the reference keeps r up to date
// by scattering A e instead, the same numbers in another order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mkb {

// one block of an aggregate: its states, its rows of A and its dense inverse
struct AggBlock {
    std::int64_t state0 = 0; // offset of the block's states in the level's state list
    std::int64_t inv0 = 0;   // offset of its n x n inverse (row-major)
    int n = 0;
    int pad = 0;
};

// blocks [agg_ptr[a], agg_ptr[a + 1]) of aggregate a; the states of block b at
// states[state0 .. state0 + n); the row of A of the state at position k of the state list is
// row_val/row_col[row_ptr[k] .. row_ptr[k + 1])
template <typename T>
struct AggView {
    const AggBlock *blocks = nullptr;
    const int *states = nullptr;
    const std::int64_t *row_ptr = nullptr;
    const int *row_col = nullptr;
    const T *row_val = nullptr;
    const T *inv = nullptr;
    T *r = nullptr; // scratch: one entry per position of the state list
    T *e = nullptr; // the corrections, likewise
};

// e_b = inverse_b (rhs_b - (A x)_b) for the blocks [b0, b1) (a warp per block); then
// x[state] += e for the same blocks
template <typename T>
cudaError_t launch_aggregate_solve(const AggView<T> &v, int b0, int b1, const T *rhs, const T *x,
                                   cudaStream_t stream);
template <typename T>
cudaError_t launch_aggregate_update(const AggView<T> &v, int b0, int b1, T *x, cudaStream_t stream);

// `sweeps` weighted Jacobi sweeps x += omega (rhs - A x) / diag(A) on each dense terminal block
// (begin, n, dense A at a_offset), x from zero when from_zero; r: scratch of the level's size
struct DenseBlock {
    std::int64_t begin = 0;
    std::int64_t a_offset = 0;
    int n = 0;
    int pad = 0;
};
template <typename T>
cudaError_t launch_dense_jacobi(const DenseBlock *blocks, int n_blocks, const T *A, const T *rhs,
                                T *x, T *r, T omega, int sweeps, bool from_zero,
                                cudaStream_t stream);

} // namespace mkb
