// sm_100a row kernels: the matrix-free generator gather and every multigrid pass built on it.
// All of them are HBM-bound gathers (no dense contraction, so no tensor cores): each thread
// unranks its state, visits its in-jumps and writes one value. Rows whose in-jumps fan in
// from every voxel take a warp (tile kind 1) or a whole block (kind 2) each. The pass (SpMV,
// residual, smoother sweep, transfer) is a launch parameter, uniform across the grid.
// Instantiated per precision in row_kernels_f64.cu and row_kernels_f32.cu.
#pragma once

#include "launch_count.hpp"
#include "row_kernels.cuh"

namespace mkb {
namespace detail {

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

template <typename T, int NS, int TMAX>
__device__ __forceinline__ void finish_row(const RowParams<T> &p, const SectorDesc &sec,
                                           std::int64_t local, const RowState<NS, TMAX> &st,
                                           T exit, T leak, T in, T in2) {
    const std::int64_t i = sec.begin + local;
    switch (p.mode) {
    case kIluPivot:
        p.y[i] = p.shift + exit - in;
        break;
    case kIluFirst: {
        const T d = p.shift + exit;
        p.aux[i] = (p.b[i] - (d * p.x[i] - in)) / d;
        break;
    }
    case kIluSecond: {
        const T xi = p.x[i];
        const T z = (p.b[i] - ((p.shift + exit) * xi - in) + in2) / p.piv[i];
        p.aux[i] = z;
        p.y[i] = xi + z;
        break;
    }
    case kIluThird:
        p.y[i] = p.x[i] + p.aux[i] + in2 / (p.shift + exit);
        break;
    case kApplyQ:
        p.y[i] = in - exit * p.x[i];
        break;
    case kApplyShifted:
        p.y[i] = (p.shift + exit) * p.x[i] - in;
        break;
    case kResidual:
        p.y[i] = p.b[i] - ((p.shift + exit) * p.x[i] - in);
        break;
    case kJacobiZero:
        p.y[i] = p.omega * p.b[i] / (p.shift + exit);
        break;
    case kJacobi: {
        const T d = p.shift + exit;
        const T xi = p.x[i];
        p.y[i] = xi + p.omega * (p.b[i] - (d * xi - in)) / d;
        break;
    }
    case kGaussSeidel:
        p.y[i] = (p.b[i] + in) / (p.shift + exit);
        break;
    case kExitLeak:
        p.y[i] = exit;
        p.aux[i] = leak;
        break;
    case kResidualRestrict: {
        const T r = p.b[i] - ((p.shift + exit) * p.x[i] - in);
        if (sec.coarse >= 0) {
            atomicAdd(p.coarse + coarse_index<NS, TMAX>(p.B, p.tv, sec, p.md.V, st, nullptr), r);
        } else {
            p.aux[i] = r;
        }
        break;
    }
    case kDiagonal:
        p.y[i] = p.shift + exit;
        break;
    default:
        break;
    }
}

template <typename T, int NS, int TMAX>
__device__ __forceinline__ void transfer_row(const RowParams<T> &p, const SectorDesc &sec,
                                             std::int64_t local, const RowState<NS, TMAX> &st) {
    const std::int64_t i = sec.begin + local;
    if (sec.coarse < 0) {
        if (p.mode == kProlong) {
            p.y[i] = T(0);
        }
        return;
    }
    if (p.mode == kRestrict) {
        atomicAdd(p.coarse + coarse_index<NS, TMAX>(p.B, p.tv, sec, p.md.V, st, nullptr), p.x[i]);
        return;
    }
    double w = 0.0;
    const std::int64_t c = coarse_index<NS, TMAX>(p.B, p.tv, sec, p.md.V, st, &w);
    if (p.mode == kProlongAdd) {
        p.y[i] += static_cast<T>(w) * p.coarse[c];
    } else {
        p.y[i] = static_cast<T>(w) * p.coarse[c];
    }
}

__device__ __forceinline__ bool is_transfer(int mode) {
    return mode == kProlongAdd || mode == kProlong || mode == kRestrict;
}
__device__ __forceinline__ bool needs_in(int mode) {
    return !(mode == kJacobiZero || mode == kExitLeak || mode == kDiagonal);
}

// the colour a pass visits (-1: every row)
__device__ __forceinline__ int pass_colour(int mode, int colour) {
    switch (mode) {
    case kGaussSeidel:
        return colour;
    case kIluFirst:
    case kIluThird:
        return 0;
    case kIluPivot:
    case kIluSecond:
        return 1;
    default:
        return -1;
    }
}

// the terms of one row computed by `nlanes` cooperating threads; lane 0 takes the light terms
template <typename T, int NS, int TMAX>
__device__ __forceinline__ void row_terms(const RowParams<T> &p, const SectorDesc &sec,
                                          std::int64_t local, const RowState<NS, TMAX> &st,
                                          int lane, int nlanes, T &exit, T &leak, T &in, T &in2) {
    if (!needs_in(p.mode)) {
        visit_row<T, NS, TMAX, false>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane,
                                      nlanes, exit, leak, [&](int, T, T) {});
        return;
    }
    if (p.mode == kIluPivot) {
        // sum over in-jumps of rate(j -> i) rate(i -> j) / diagonal_j (aux holds the diagonal)
        const T *dg = p.aux;
        visit_row<T, NS, TMAX, true, true>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane,
                                           nlanes, exit, leak,
                                           [&](int j, T a, T rev) { in += a * rev / dg[j]; });
        return;
    }
    // Gauss-Seidel and the ILU passes update x (= y) in place: rows of one colour read only
    // the other colour's entries, through plain coherent loads
    const int mode = p.mode;
    const T *xs = mode == kGaussSeidel ? p.y : p.x;
    const T *ax = p.aux;
    visit_row<T, NS, TMAX, true>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane, nlanes,
                                 exit, leak, [&](int j, T a, T) {
                                     if (mode == kIluThird) {
                                         in2 += a * ax[j];
                                         return;
                                     }
                                     in += a * xs[j];
                                     if (mode == kIluSecond) {
                                         in2 += a * ax[j];
                                     }
                                 });
}

template <typename T, int NS, int TMAX>
__global__ void __launch_bounds__(kRowBlock) row_kernel(const __grid_constant__ RowParams<T> p) {
    __shared__ SectorDesc s_sec;
    __shared__ T s_red[4][kRowBlock / 32];
    const Tile tile = p.tiles[blockIdx.x];
    if (threadIdx.x == 0) {
        s_sec = p.sectors[tile.sector];
    }
    __syncthreads();
    const SectorDesc &sec = s_sec;
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x) & 31;

    std::int64_t local;
    int row_lane, row_lanes;
    if (tile.kind == 0) {
        if (static_cast<int>(threadIdx.x) >= tile.count) {
            return;
        }
        local = tile.local0 + threadIdx.x;
        row_lane = 0;
        row_lanes = 1;
    } else if (tile.kind == 1) {
        if (warp >= tile.count) {
            return;
        }
        local = tile.local0 + warp;
        row_lane = lane;
        row_lanes = 32;
    } else {
        local = tile.local0;
        row_lane = static_cast<int>(threadIdx.x);
        row_lanes = kRowBlock;
    }
    RowState<NS, TMAX> st;
    load_state<NS, TMAX>(p.B, sec, p.md.S, p.md.V, local, st);
    if (is_transfer(p.mode)) {
        if (row_lane == 0) {
            transfer_row<T, NS, TMAX>(p, sec, local, st);
        }
        return;
    }
    const int colour = pass_colour(p.mode, p.colour);
    if (colour >= 0 && state_colour<T, NS, TMAX>(p.md, sec, st) != colour) {
        return; // uniform across the warp or block of a shared row
    }
    T exit = T(0), leak = T(0), in = T(0), in2 = T(0);
    row_terms<T, NS, TMAX>(p, sec, local, st, row_lane, row_lanes, exit, leak, in, in2);
    if (tile.kind == 0) {
        finish_row<T, NS, TMAX>(p, sec, local, st, exit, leak, in, in2);
        return;
    }
    exit = warp_sum(exit);
    leak = warp_sum(leak);
    in = warp_sum(in);
    in2 = warp_sum(in2);
    if (tile.kind == 1) {
        if (lane == 0) {
            finish_row<T, NS, TMAX>(p, sec, local, st, exit, leak, in, in2);
        }
        return;
    }
    if (lane == 0) {
        s_red[0][warp] = exit;
        s_red[1][warp] = leak;
        s_red[2][warp] = in;
        s_red[3][warp] = in2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        exit = leak = in = in2 = T(0);
        for (int w = 0; w < kRowBlock / 32; ++w) {
            exit += s_red[0][w];
            leak += s_red[1][w];
            in += s_red[2][w];
            in2 += s_red[3][w];
        }
        finish_row<T, NS, TMAX>(p, sec, local, st, exit, leak, in, in2);
    }
}

template <typename T, int NS, int TMAX>
cudaError_t launch_shape(const RowParams<T> &p, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    count_launches(1);
    row_kernel<T, NS, TMAX><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

} // namespace detail

// (species, largest species total) -> the instantiated state shape
template <typename T>
cudaError_t launch_rows_impl(const RowParams<T> &p, int S, int cap, cudaStream_t stream) {
    return with_shape(S, cap, [&]<int NS, int TMAX>() {
        return detail::launch_shape<T, NS, TMAX>(p, stream);
    });
}

} // namespace mkb
