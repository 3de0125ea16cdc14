// sm_100a row kernels: the matrix-free generator gather and every multigrid pass built on it.
// Each thread unranks its state, visits its in-jumps and writes one value per column. Rows
// whose in-jumps fan in from every voxel take a warp (tile kind 1) or a whole block (kind 2)
// each. The pass (SpMV, residual, smoother sweep, multigrid set-up) is a launch parameter,
// uniform across the grid. NB > 1 instantiations serve up to NB right-hand sides at once
// (columns at stride ldv): the ranking and rate work of a row, which bounds these kernels, is
// done once for all columns.
// Instantiated once per (precision, batch width, state shape) by row_kernels_inst.cu, so the
// shapes compile in parallel; row_kernels.cu dispatches to them.
#pragma once

#include "launch_count.hpp"
#include "row_kernels.cuh"

#include <type_traits>

namespace mkb {
namespace detail {

// The FP32 kernels that serve kRowBatch right-hand sides (the batched multigrid cycle) keep
// them interleaved: element (i, c) at i * kRowBatch + c, so an in-jump's kRowBatch source
// values are one 16-byte load. They compute every lane; lanes at or above p.nb hold zeros.
// The other batched kernels keep column c at c * ldv.
template <typename T, int NB>
constexpr bool kInterleaved = std::is_same_v<T, float> && NB == kRowBatch && kRowBatch == 4;

template <typename T, int NB>
__device__ __forceinline__ std::int64_t at(std::int64_t i, int c, std::int64_t ld) {
    if constexpr (kInterleaved<T, NB>) {
        return i * NB + c;
    } else {
        return i + c * ld;
    }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

// the diagonal of column c: its shift plus the row's exit rate
template <typename T>
__device__ __forceinline__ T column_shift(const RowParams<T> &p, int c) {
    return p.per_col_shift ? p.col_shift[c] : p.shift;
}

// write one row's result for each column from its accumulated terms; every pass writes rows
// of its own tile only, so results do not depend on how rows are spread over blocks. MODE >= 0
// fixes the pass at compile time (else p.mode selects it).
template <typename T, int NB, int MODE = -1>
__device__ __forceinline__ void finish_row(const RowParams<T> &p, std::int64_t i, T exit, T leak,
                                           const T (&in)[NB], const T (&in2)[NB]) {
    const int mode = MODE >= 0 ? MODE : p.mode;
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        if (!kInterleaved<T, NB> && c >= p.nb) {
            break;
        }
        const T d = column_shift(p, c) + exit;
        const std::int64_t k = at<T, NB>(i, c, p.ldv);
        switch (mode) {
        case kIluPivot:
            p.y[k] = d - in[c];
            break;
        case kIluFirst:
            p.aux[k] = (p.b[k] - (d * p.x[k] - in[c])) / d;
            break;
        case kIluSecond: {
            const T xi = p.x[k];
            const T z = (p.b[k] - (d * xi - in[c]) + in2[c]) / p.piv[p.piv_per_col ? k : i];
            p.aux[k] = z;
            p.y[k] = xi + z;
            break;
        }
        case kIluThird:
            p.y[k] = p.x[k] + p.aux[k] + in2[c] / d;
            break;
        case kApplyQ:
            p.y[k] = in[c] - exit * p.x[k];
            break;
        case kApplyShifted:
            p.y[k] = d * p.x[k] - in[c];
            break;
        case kResidual:
            p.y[k] = p.b[k] - (d * p.x[k] - in[c]);
            break;
        case kJacobiZero:
            p.y[k] = p.omega * p.b[k] / d;
            break;
        case kJacobi: {
            const T xi = p.x[k];
            p.y[k] = xi + p.omega * (p.b[k] - (d * xi - in[c])) / d;
            break;
        }
        case kGaussSeidel:
            p.y[k] = (p.b[k] + in[c]) / d;
            break;
        case kExitLeak:
            p.y[k] = exit;
            p.aux[k] = leak;
            break;
        case kDiagonal:
            p.y[k] = d;
            break;
        default:
            break;
        }
    }
}

// multigrid set-up: the coarse state of a fine state and its prolongation weight
template <typename T, int NS, int TMAX>
__device__ __forceinline__ void coarse_index_row(const RowParams<T> &p, const SectorDesc &sec,
                                                 std::int64_t local, const RowState<NS, TMAX> &st) {
    const std::int64_t i = sec.begin + local;
    if (sec.coarse < 0) {
        p.idx[i] = -1;
        p.wout[i] = 0.0;
        return;
    }
    double w = 0.0;
    p.idx[i] = static_cast<int>(coarse_index<NS, TMAX>(p.B, p.tv, sec, p.md.V, st, &w));
    p.wout[i] = w;
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
template <typename T, int NS, int TMAX, int NB>
__device__ __forceinline__ void row_terms(const RowParams<T> &p, const SectorDesc &sec,
                                          std::int64_t local, const RowState<NS, TMAX> &st,
                                          int lane, int nlanes, T &exit, T &leak, T (&in)[NB],
                                          T (&in2)[NB]) {
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
                                           [&](int j, T a, T rev) { in[0] += a * rev / dg[j]; });
        return;
    }
    // Gauss-Seidel and the ILU passes update x (= y) in place: rows of one colour read only
    // the other colour's entries, through plain coherent loads
    const int mode = p.mode, nb = p.nb;
    const std::int64_t ldv = p.ldv;
    const T *xs = mode == kGaussSeidel ? p.y : p.x;
    const T *ax = p.aux;
    if constexpr (NB == 1) {
        // one column: the common passes gather x alone, with 32-bit indices
        if (mode != kIluSecond && mode != kIluThird) {
            visit_row<T, NS, TMAX, true>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane,
                                         nlanes, exit, leak,
                                         [&](int j, T a, T) { in[0] += a * xs[j]; });
            return;
        }
    }
    if constexpr (kInterleaved<T, NB>) {
        // the kRowBatch source values of an in-jump in one 16-byte load
        visit_row<T, NS, TMAX, true>(
            p.B, p.sectors, sec, p.md, local, st, lane == 0, lane, nlanes, exit, leak,
            [&](int j, T a, T) {
                const std::int64_t k = static_cast<std::int64_t>(j) * NB;
                if (mode != kIluThird) {
                    const float4 v = *reinterpret_cast<const float4 *>(xs + k);
                    in[0] += a * v.x;
                    in[1] += a * v.y;
                    in[2] += a * v.z;
                    in[3] += a * v.w;
                }
                if (mode == kIluSecond || mode == kIluThird) {
                    const float4 u = *reinterpret_cast<const float4 *>(ax + k);
                    in2[0] += a * u.x;
                    in2[1] += a * u.y;
                    in2[2] += a * u.z;
                    in2[3] += a * u.w;
                }
            });
        return;
    }
    visit_row<T, NS, TMAX, true>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane, nlanes,
                                 exit, leak, [&](int j, T a, T) {
#pragma unroll
                                     for (int c = 0; c < NB; ++c) {
                                         if (c >= nb) {
                                             break;
                                         }
                                         const std::int64_t k = j + c * ldv;
                                         if (mode == kIluThird) {
                                             in2[c] += a * ax[k];
                                             continue;
                                         }
                                         in[c] += a * xs[k];
                                         if (mode == kIluSecond) {
                                             in2[c] += a * ax[k];
                                         }
                                     }
                                 });
}

template <typename T, int NS, int TMAX, int NB>
__global__ void __launch_bounds__(kRowBlock) row_kernel(const __grid_constant__ RowParams<T> p) {
    __shared__ SectorDesc s_sec;
    __shared__ T s_red[2 + 2 * NB][kRowBlock / 32];
    const Tile tile = p.tiles[blockIdx.x];
    if (threadIdx.x == 0) {
        s_sec = p.sectors[tile.sector];
    }
    __syncthreads();
    const SectorDesc &sec = s_sec;
    if (p.sector_class >= 0 && sec.gs_class != p.sector_class) {
        return; // another colour class's pass (the whole block)
    }
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
    if (p.mode == kCoarseIndex) {
        if (row_lane == 0) {
            coarse_index_row<T, NS, TMAX>(p, sec, local, st);
        }
        return;
    }
    const int colour = pass_colour(p.mode, p.colour);
    if (colour >= 0 && state_colour<T, NS, TMAX>(p.md, sec, st) != colour) {
        return; // uniform across the warp or block of a shared row
    }
    T exit = T(0), leak = T(0);
    T in[NB], in2[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] = T(0);
        in2[c] = T(0);
    }
    row_terms<T, NS, TMAX, NB>(p, sec, local, st, row_lane, row_lanes, exit, leak, in, in2);
    if (tile.kind == 0) {
        finish_row<T, NB>(p, sec.begin + local, exit, leak, in, in2);
        return;
    }
    exit = warp_sum(exit);
    leak = warp_sum(leak);
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] = warp_sum(in[c]);
        in2[c] = warp_sum(in2[c]);
    }
    if (tile.kind == 1) {
        if (lane == 0) {
            finish_row<T, NB>(p, sec.begin + local, exit, leak, in, in2);
        }
        return;
    }
    if (lane == 0) {
        s_red[0][warp] = exit;
        s_red[1][warp] = leak;
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            s_red[2 + c][warp] = in[c];
            s_red[2 + NB + c][warp] = in2[c];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        exit = leak = T(0);
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            in[c] = in2[c] = T(0);
        }
        for (int w = 0; w < kRowBlock / 32; ++w) {
            exit += s_red[0][w];
            leak += s_red[1][w];
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                in[c] += s_red[2 + c][w];
                in2[c] += s_red[2 + NB + c][w];
            }
        }
        finish_row<T, NB>(p, sec.begin + local, exit, leak, in, in2);
    }
}

template <typename T, int NS, int TMAX, int NB>
cudaError_t launch_shape(const RowParams<T> &p, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    count_launches(1);
    row_kernel<T, NS, TMAX, NB><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

} // namespace detail
} // namespace mkb
