// Kernels of the aggregate-block smoother and of the dense-block Jacobi sweeps (aggregate.cuh).
#include "aggregate.cuh"
#include "launch_count.hpp"

#include <algorithm>

namespace mkb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// a warp per block: the lanes form the block's residual entries r, then the rows of inverse * r
template <typename T>
__global__ void __launch_bounds__(kThreads)
    aggregate_solve_kernel(const AggView<T> v, int b0, int b1, const T *rhs, const T *x) {
    const int warp = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int b = b0 + static_cast<int>(blockIdx.x) * kWarps + warp;
    if (b >= b1) {
        return;
    }
    const AggBlock blk = v.blocks[b];
    const int *st = v.states + blk.state0;
    for (int k = lane; k < blk.n; k += 32) {
        const std::int64_t pos = blk.state0 + k;
        T ax = T(0);
        for (std::int64_t q = v.row_ptr[pos]; q < v.row_ptr[pos + 1]; ++q) {
            ax += v.row_val[q] * x[v.row_col[q]];
        }
        v.r[pos] = rhs[st[k]] - ax;
    }
    __syncwarp();
    const T *inv = v.inv + blk.inv0;
    const T *r = v.r + blk.state0;
    for (int k = lane; k < blk.n; k += 32) {
        const T *row = inv + static_cast<std::int64_t>(k) * blk.n;
        T s = T(0);
        for (int q = 0; q < blk.n; ++q) {
            s += row[q] * r[q];
        }
        v.e[blk.state0 + k] = s;
    }
}

template <typename T>
__global__ void aggregate_update_kernel(const AggView<T> v, int b0, int b1, T *x) {
    const int warp = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    const int b = b0 + static_cast<int>(blockIdx.x) * kWarps + warp;
    if (b >= b1) {
        return;
    }
    const AggBlock blk = v.blocks[b];
    for (int k = lane; k < blk.n; k += 32) {
        x[v.states[blk.state0 + k]] += v.e[blk.state0 + k];
    }
}

// a CUDA block per dense block; the sweeps separated by block barriers
template <typename T>
__global__ void __launch_bounds__(kThreads)
    dense_jacobi_kernel(const DenseBlock *blocks, const T *A, const T *rhs, T *x, T *r, T omega,
                        int sweeps, bool from_zero) {
    const DenseBlock blk = blocks[blockIdx.x];
    const int n = blk.n;
    const T *a = A + blk.a_offset;
    T *xb = x + blk.begin;
    T *rb = r + blk.begin;
    const T *bb = rhs + blk.begin;
    if (from_zero) {
        for (int p = static_cast<int>(threadIdx.x); p < n; p += kThreads) {
            xb[p] = T(0);
        }
        __syncthreads();
    }
    for (int s = 0; s < sweeps; ++s) {
        for (int p = static_cast<int>(threadIdx.x); p < n; p += kThreads) {
            const T *row = a + static_cast<std::int64_t>(p) * n;
            T ax = T(0);
            for (int q = 0; q < n; ++q) {
                ax += row[q] * xb[q];
            }
            rb[p] = bb[p] - ax;
        }
        __syncthreads();
        for (int p = static_cast<int>(threadIdx.x); p < n; p += kThreads) {
            xb[p] += omega * rb[p] / a[static_cast<std::int64_t>(p) * n + p];
        }
        __syncthreads();
    }
}

unsigned warp_blocks(int blocks) { return static_cast<unsigned>((blocks + kWarps - 1) / kWarps); }

} // namespace

template <typename T>
cudaError_t launch_aggregate_solve(const AggView<T> &v, int b0, int b1, const T *rhs, const T *x,
                                   cudaStream_t stream) {
    if (b1 <= b0) {
        return cudaSuccess;
    }
    count_launches(1);
    aggregate_solve_kernel<T><<<warp_blocks(b1 - b0), kThreads, 0, stream>>>(v, b0, b1, rhs, x);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_aggregate_update(const AggView<T> &v, int b0, int b1, T *x, cudaStream_t stream) {
    if (b1 <= b0) {
        return cudaSuccess;
    }
    count_launches(1);
    aggregate_update_kernel<T><<<warp_blocks(b1 - b0), kThreads, 0, stream>>>(v, b0, b1, x);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_dense_jacobi(const DenseBlock *blocks, int n_blocks, const T *A, const T *rhs,
                                T *x, T *r, T omega, int sweeps, bool from_zero,
                                cudaStream_t stream) {
    if (n_blocks == 0 || (sweeps == 0 && !from_zero)) {
        return cudaSuccess;
    }
    count_launches(1);
    dense_jacobi_kernel<T><<<n_blocks, kThreads, 0, stream>>>(blocks, A, rhs, x, r, omega, sweeps,
                                                              from_zero);
    return cudaGetLastError();
}

template cudaError_t launch_aggregate_solve<double>(const AggView<double> &, int, int, const double *,
                                                    const double *, cudaStream_t);
template cudaError_t launch_aggregate_solve<float>(const AggView<float> &, int, int, const float *,
                                                   const float *, cudaStream_t);
template cudaError_t launch_aggregate_update<double>(const AggView<double> &, int, int, double *,
                                                     cudaStream_t);
template cudaError_t launch_aggregate_update<float>(const AggView<float> &, int, int, float *,
                                                    cudaStream_t);
template cudaError_t launch_dense_jacobi<double>(const DenseBlock *, int, const double *, const double *,
                                                 double *, double *, double, int, bool, cudaStream_t);
template cudaError_t launch_dense_jacobi<float>(const DenseBlock *, int, const float *, const float *,
                                                float *, float *, float, int, bool, cudaStream_t);

} // namespace mkb
