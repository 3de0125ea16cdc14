// Dispatch of the row kernels (the general kernel instantiated per shape by
// row_kernels_inst.cu, the stencil kernel by stencil_rows.cu), the dense terminal solve of the
// multigrid, and bit-exact state indexing on the device.
#include "launch_count.hpp"
#include "row_kernels.cuh"

#include <algorithm>

namespace mkb {

int mol_cap_for(int n_species, int max_species_total) {
    const int limit = n_species == 1 ? 64 : 16;
    if (max_species_total > limit) {
        return -1;
    }
    for (int cap : {1, 2, 4, 16, 64}) {
        if (max_species_total <= cap) {
            return cap;
        }
    }
    return -1;
}

namespace {

// (species, largest species total) -> the general kernel of that state shape
template <typename T, int NB>
cudaError_t launch_general(const RowParams<T> &p, int S, int cap, cudaStream_t stream) {
    return with_shape(S, cap, [&]<int NS, int TMAX>() {
        return detail::launch_shape<T, NS, TMAX, NB>(p, stream);
    });
}

} // namespace

cudaError_t launch_rows_f64(const RowParams<double> &p, int S, int cap, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? launch_general<double, kRowBatch>(p, S, cap, stream)
                    : launch_general<double, 1>(p, S, cap, stream);
}

cudaError_t launch_rows_f32(const RowParams<float> &p, int S, int cap, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? launch_general<float, kRowBatch>(p, S, cap, stream)
                    : launch_general<float, 1>(p, S, cap, stream);
}

template <>
cudaError_t launch_rows<double>(RowMode mode, int S, int cap, const RowParams<double> &p,
                                cudaStream_t stream) {
    RowParams<double> q = p;
    q.mode = mode;
    return launch_rows_f64(q, S, cap, stream);
}

template <>
cudaError_t launch_rows<float>(RowMode mode, int S, int cap, const RowParams<float> &p,
                               cudaStream_t stream) {
    RowParams<float> q = p;
    q.mode = mode;
    return launch_rows_f32(q, S, cap, stream);
}

bool stencil_shape(int S, int cap) { return (S == 1 && cap <= 4) || (S == 2 && cap <= 1); }

bool stencil_mode(int mode) {
    switch (mode) {
    case kApplyQ:
    case kApplyShifted:
    case kResidual:
    case kJacobiZero:
    case kJacobi:
    case kGaussSeidel:
    case kIluFirst:
    case kIluSecond:
    case kIluThird:
        return true;
    default:
        return false;
    }
}

cudaError_t launch_stencil_rows_f64(const RowParams<double> &p, int S, int cap,
                                    cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !stencil_shape(S, cap) || !stencil_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_stencil<double, kRowBatch>(p, S, cap, stream)
                    : detail::launch_stencil<double, 1>(p, S, cap, stream);
}

cudaError_t launch_stencil_rows_f32(const RowParams<float> &p, int S, int cap,
                                    cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !stencil_shape(S, cap) || !stencil_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_stencil<float, kRowBatch>(p, S, cap, stream)
                    : detail::launch_stencil<float, 1>(p, S, cap, stream);
}

bool pair_heavy_mode(int mode) { return mode == kApplyQ || mode == kApplyShifted || mode == kResidual; }

cudaError_t launch_pair_heavy_rows_f64(const RowParams<double> &p, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !pair_heavy_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_pair_heavy<double, kRowBatch>(p, stream)
                    : detail::launch_pair_heavy<double, 1>(p, stream);
}

cudaError_t launch_pair_heavy_rows_f32(const RowParams<float> &p, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !pair_heavy_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_pair_heavy<float, kRowBatch>(p, stream)
                    : detail::launch_pair_heavy<float, 1>(p, stream);
}

cudaError_t launch_pair_strip_rows_f64(const RowParams<double> &p, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !stencil_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_pair_strip<double, kRowBatch>(p, stream)
                    : detail::launch_pair_strip<double, 1>(p, stream);
}

cudaError_t launch_pair_strip_rows_f32(const RowParams<float> &p, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !stencil_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_pair_strip<float, kRowBatch>(p, stream)
                    : detail::launch_pair_strip<float, 1>(p, stream);
}

cudaError_t launch_pair_heavy_group_rows_f64(const RowParams<double> &p, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !pair_heavy_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_pair_heavy_group<double, kRowBatch>(p, stream)
                    : detail::launch_pair_heavy_group<double, 1>(p, stream);
}

cudaError_t launch_pair_heavy_group_rows_f32(const RowParams<float> &p, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch || !pair_heavy_mode(p.mode)) {
        return cudaErrorInvalidValue;
    }
    return p.nb > 1 ? detail::launch_pair_heavy_group<float, kRowBatch>(p, stream)
                    : detail::launch_pair_heavy_group<float, 1>(p, stream);
}

namespace {

constexpr int kTerminalThreads = 256;

// x[begin + p] += inv[p] . r[begin ..]: one warp per row of a block's inverse, the lanes
// striding its columns (coalesced); blockIdx.x picks the terminal block, blockIdx.y a group of
// rows, so a large block's rows spread over many SMs. Entry q of r and x sits at q * stride
// (stride > 1: one column of interleaved right-hand sides).
template <typename T>
__global__ void __launch_bounds__(kTerminalThreads)
    terminal_kernel(const TerminalBlock *blocks, const T *inv, const T *r, T *x, int stride) {
    const TerminalBlock tb = blocks[blockIdx.x];
    constexpr int warps = kTerminalThreads / 32;
    const int warp = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    for (int p = static_cast<int>(blockIdx.y) * warps + warp; p < tb.n;
         p += static_cast<int>(gridDim.y) * warps) {
        const T *row = inv + tb.inv_offset + static_cast<std::int64_t>(p) * tb.n;
        T e = T(0);
        for (int q = lane; q < tb.n; q += 32) {
            e += row[q] * r[(tb.begin + q) * stride];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, off);
        }
        if (lane == 0) {
            x[(tb.begin + p) * stride] += e;
        }
    }
}

__device__ int find_sector_of(const SectorDesc *sectors, int n_sectors, std::int64_t i) {
    int lo = 0, hi = n_sectors - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sectors[mid].begin <= i) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

constexpr int kIndexCap = 64;

__global__ void unrank_kernel(const BinomTable B, const SectorDesc *sectors, int n_sectors, int S,
                              int V, const std::int64_t *index, std::int64_t count, int *states) {
    const std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
    if (t >= count) {
        return;
    }
    int *out = states + t * static_cast<std::int64_t>(V) * S;
    for (std::int64_t k = 0; k < static_cast<std::int64_t>(V) * S; ++k) {
        out[k] = 0;
    }
    const std::int64_t i = index[t];
    if (i < 0) {
        return;
    }
    const int k = find_sector_of(sectors, n_sectors, i);
    const SectorDesc &sec = sectors[k];
    if (i >= sec.begin + sec.size) {
        return;
    }
    std::int64_t rank[kMaxSpecies];
    split_local(sec, S, i - sec.begin, rank);
    int u[kIndexCap];
    for (int s = 0; s < S; ++s) {
        unrank_species<kIndexCap>(B, rank[s], sec.total[s], V, u);
        for (int q = 0; q < sec.total[s]; ++q) {
            out[static_cast<std::int64_t>(V - 1 - u[q]) * S + s] += 1;
        }
    }
}

__global__ void rank_kernel(const BinomTable B, const SectorDesc *sectors, int n_sectors,
                            const int *max_totals, int is_box, int S, int V, const int *states,
                            std::int64_t count, std::int64_t *index) {
    const std::int64_t t = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
    if (t >= count) {
        return;
    }
    const int *x = states + t * static_cast<std::int64_t>(V) * S;
    int totals[kMaxSpecies] = {};
    for (int v = 0; v < V; ++v) {
        for (int s = 0; s < S; ++s) {
            const int c = x[static_cast<std::int64_t>(v) * S + s];
            if (c < 0) {
                index[t] = -1;
                return;
            }
            totals[s] += c;
        }
    }
    int k = 0;
    if (is_box) {
        for (int s = 0; s < S; ++s) {
            if (totals[s] > max_totals[s]) {
                index[t] = -1;
                return;
            }
            k = k * (max_totals[s] + 1) + totals[s];
        }
    } else {
        for (int s = 0; s < S; ++s) {
            if (totals[s] != sectors[0].total[s]) {
                index[t] = -1;
                return;
            }
        }
    }
    if (k >= n_sectors) {
        index[t] = -1;
        return;
    }
    const SectorDesc &sec = sectors[k];
    std::int64_t local = 0;
    int u[kIndexCap];
    for (int s = 0; s < S; ++s) {
        if (totals[s] > kIndexCap) {
            index[t] = -1;
            return;
        }
        int n = 0;
        for (int v = V - 1; v >= 0; --v) {
            const int c = x[static_cast<std::int64_t>(v) * S + s];
            for (int q = 0; q < c; ++q) {
                u[n++] = V - 1 - v;
            }
        }
        local += rank_species<kIndexCap>(B, u, n) * sec.stride[s];
    }
    index[t] = sec.begin + local;
}

} // namespace

template <typename T>
cudaError_t launch_terminal(const TerminalBlock *blocks, int n_blocks, int max_n, const T *inv,
                            const T *r, T *x, int stride, cudaStream_t stream) {
    if (n_blocks == 0) {
        return cudaSuccess;
    }
    constexpr int warps = kTerminalThreads / 32;
    const int groups = std::max(1, std::min((max_n + warps - 1) / warps, 256));
    count_launches(1);
    terminal_kernel<T>
        <<<dim3(n_blocks, groups), kTerminalThreads, 0, stream>>>(blocks, inv, r, x, stride);
    return cudaGetLastError();
}

template cudaError_t launch_terminal<double>(const TerminalBlock *, int, int, const double *,
                                             const double *, double *, int, cudaStream_t);
template cudaError_t launch_terminal<float>(const TerminalBlock *, int, int, const float *,
                                            const float *, float *, int, cudaStream_t);

cudaError_t launch_unrank(const BinomTable &B, const SectorDesc *sectors, int n_sectors, int S,
                          int V, const std::int64_t *index, std::int64_t count, int *states,
                          cudaStream_t stream) {
    if (count == 0) {
        return cudaSuccess;
    }
    const int threads = 128;
    const auto blocks = static_cast<unsigned>((count + threads - 1) / threads);
    count_launches(1);
    unrank_kernel<<<blocks, threads, 0, stream>>>(B, sectors, n_sectors, S, V, index, count,
                                                  states);
    return cudaGetLastError();
}

cudaError_t launch_rank(const BinomTable &B, const SectorDesc *sectors, int n_sectors,
                        const int *max_totals, int is_box, int S, int V, const int *states,
                        std::int64_t count, std::int64_t *index, cudaStream_t stream) {
    if (count == 0) {
        return cudaSuccess;
    }
    const int threads = 128;
    const auto blocks = static_cast<unsigned>((count + threads - 1) / threads);
    count_launches(1);
    rank_kernel<<<blocks, threads, 0, stream>>>(B, sectors, n_sectors, max_totals, is_box, S, V,
                                                states, count, index);
    return cudaGetLastError();
}

} // namespace mkb
