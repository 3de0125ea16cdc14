// sm_100a row kernels: the matrix-free generator gather and every multigrid pass built on it.
// All of them are HBM-bound gathers (no dense contraction, so no tensor cores): each
// thread unranks its state, visits its in-jumps and writes one value.
#include "row_kernels.cuh"

namespace mkb {

int mol_cap_for(int n_mol) {
    for (int cap : kMolCaps) {
        if (n_mol <= cap) {
            return cap;
        }
    }
    return -1;
}

namespace {

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

template <typename T, int MAXM, int MODE>
__device__ __forceinline__ void finish_row(const RowParams<T> &p, const SectorDesc &sec,
                                           std::int64_t local, const RowState<MAXM> &st, T exit,
                                           T leak, T in) {
    const std::int64_t i = sec.begin + local;
    if constexpr (MODE == kApplyQ) {
        p.y[i] = in - exit * p.x[i];
    } else if constexpr (MODE == kApplyShifted) {
        p.y[i] = (p.shift + exit) * p.x[i] - in;
    } else if constexpr (MODE == kResidual) {
        p.y[i] = p.b[i] - ((p.shift + exit) * p.x[i] - in);
    } else if constexpr (MODE == kJacobiZero) {
        p.y[i] = p.omega * p.b[i] / (p.shift + exit);
    } else if constexpr (MODE == kJacobi) {
        const T d = p.shift + exit;
        const T xi = p.x[i];
        p.y[i] = xi + p.omega * (p.b[i] - (d * xi - in)) / d;
    } else if constexpr (MODE == kGaussSeidel) {
        p.y[i] = (p.b[i] + in) / (p.shift + exit);
    } else if constexpr (MODE == kExitLeak) {
        p.y[i] = exit;
        p.aux[i] = leak;
    } else if constexpr (MODE == kResidualRestrict) {
        const T r = p.b[i] - ((p.shift + exit) * p.x[i] - in);
        if (sec.coarse >= 0) {
            const std::int64_t c =
                coarse_index<MAXM>(p.B, p.tv, sec, p.md.S, p.md.V, st, nullptr);
            atomicAdd(p.coarse + c, r);
        } else {
            p.aux[i] = r;
        }
    } else if constexpr (MODE == kDiagonal) {
        p.y[i] = p.shift + exit;
    }
}

template <typename T, int MAXM, int MODE>
__device__ __forceinline__ void transfer_row(const RowParams<T> &p, const SectorDesc &sec,
                                             std::int64_t local, const RowState<MAXM> &st) {
    const std::int64_t i = sec.begin + local;
    if (sec.coarse < 0) {
        if constexpr (MODE == kProlong) {
            p.y[i] = T(0);
        }
        return;
    }
    if constexpr (MODE == kRestrict) {
        const std::int64_t c = coarse_index<MAXM>(p.B, p.tv, sec, p.md.S, p.md.V, st, nullptr);
        atomicAdd(p.coarse + c, p.x[i]);
    } else {
        double w = 0.0;
        const std::int64_t c = coarse_index<MAXM>(p.B, p.tv, sec, p.md.S, p.md.V, st, &w);
        if constexpr (MODE == kProlongAdd) {
            p.y[i] += static_cast<T>(w) * p.coarse[c];
        } else {
            p.y[i] = static_cast<T>(w) * p.coarse[c];
        }
    }
}

template <typename T, int MAXM, int MODE>
__global__ void __launch_bounds__(kRowBlock) row_kernel(const RowParams<T> p) {
    __shared__ SectorDesc s_sec;
    const Tile tile = p.tiles[blockIdx.x];
    if (threadIdx.x == 0) {
        s_sec = p.sectors[tile.sector];
    }
    __syncthreads();
    const SectorDesc &sec = s_sec;
    // in-place Gauss-Seidel reads x while other threads write it: plain loads there
    const T *xs = (MODE == kGaussSeidel) ? p.y : p.x;

    if (tile.kind == 0) {
        if (static_cast<int>(threadIdx.x) >= tile.count) {
            return;
        }
        const std::int64_t local = tile.local0 + threadIdx.x;
        RowState<MAXM> st;
        load_state<MAXM>(p.B, sec, p.md.S, p.md.V, local, st);
        if constexpr (MODE == kProlongAdd || MODE == kProlong || MODE == kRestrict) {
            transfer_row<T, MAXM, MODE>(p, sec, local, st);
            return;
        } else {
            if constexpr (MODE == kGaussSeidel) {
                if (state_colour<T, MAXM>(p.md, sec, st) != p.colour) {
                    return;
                }
            }
            T exit = T(0), leak = T(0), in = T(0);
            if constexpr (MODE == kGaussSeidel) {
                visit_row<T, MAXM>(p.B, p.sectors, sec, p.md, local, st, true, 0, 1, exit, leak,
                                   [&](std::int64_t j, T a) { in += a * xs[j]; });
            } else if constexpr (MODE == kJacobiZero || MODE == kExitLeak || MODE == kDiagonal) {
                visit_row<T, MAXM, false>(p.B, p.sectors, sec, p.md, local, st, true, 0, 1, exit,
                                          leak, [&](std::int64_t, T) {});
            } else {
                visit_row<T, MAXM>(p.B, p.sectors, sec, p.md, local, st, true, 0, 1, exit, leak,
                                   [&](std::int64_t j, T a) { in += a * __ldg(xs + j); });
            }
            finish_row<T, MAXM, MODE>(p, sec, local, st, exit, leak, in);
        }
        return;
    }

    // one warp per row: lane 0 takes the light terms, all lanes split the voxel loop
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    if (warp >= tile.count) {
        return;
    }
    const std::int64_t local = tile.local0 + warp;
    RowState<MAXM> st;
    load_state<MAXM>(p.B, sec, p.md.S, p.md.V, local, st);
    if constexpr (MODE == kProlongAdd || MODE == kProlong || MODE == kRestrict) {
        if (lane == 0) {
            transfer_row<T, MAXM, MODE>(p, sec, local, st);
        }
        return;
    } else {
        if constexpr (MODE == kGaussSeidel) {
            if (state_colour<T, MAXM>(p.md, sec, st) != p.colour) {
                return;
            }
        }
        T exit = T(0), leak = T(0), in = T(0);
        if constexpr (MODE == kGaussSeidel) {
            visit_row<T, MAXM>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane, 32, exit,
                               leak, [&](std::int64_t j, T a) { in += a * xs[j]; });
        } else if constexpr (MODE == kJacobiZero || MODE == kExitLeak || MODE == kDiagonal) {
            visit_row<T, MAXM, false>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane, 32,
                                      exit, leak, [&](std::int64_t, T) {});
        } else {
            visit_row<T, MAXM>(p.B, p.sectors, sec, p.md, local, st, lane == 0, lane, 32, exit,
                               leak, [&](std::int64_t j, T a) { in += a * __ldg(xs + j); });
        }
        exit = warp_sum(exit);
        leak = warp_sum(leak);
        in = warp_sum(in);
        if (lane == 0) {
            finish_row<T, MAXM, MODE>(p, sec, local, st, exit, leak, in);
        }
    }
}

template <typename T, int MAXM, int MODE>
cudaError_t launch_one(const RowParams<T> &p, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    row_kernel<T, MAXM, MODE><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
    return cudaGetLastError();
}

template <typename T, int MAXM>
cudaError_t launch_mode(RowMode mode, const RowParams<T> &p, cudaStream_t stream) {
    switch (mode) {
    case kApplyQ:
        return launch_one<T, MAXM, kApplyQ>(p, stream);
    case kApplyShifted:
        return launch_one<T, MAXM, kApplyShifted>(p, stream);
    case kResidual:
        return launch_one<T, MAXM, kResidual>(p, stream);
    case kJacobiZero:
        return launch_one<T, MAXM, kJacobiZero>(p, stream);
    case kJacobi:
        return launch_one<T, MAXM, kJacobi>(p, stream);
    case kGaussSeidel:
        return launch_one<T, MAXM, kGaussSeidel>(p, stream);
    case kExitLeak:
        return launch_one<T, MAXM, kExitLeak>(p, stream);
    case kResidualRestrict:
        return launch_one<T, MAXM, kResidualRestrict>(p, stream);
    case kProlongAdd:
        return launch_one<T, MAXM, kProlongAdd>(p, stream);
    case kDiagonal:
        return launch_one<T, MAXM, kDiagonal>(p, stream);
    case kRestrict:
        return launch_one<T, MAXM, kRestrict>(p, stream);
    case kProlong:
        return launch_one<T, MAXM, kProlong>(p, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

template <typename T>
__global__ void terminal_kernel(const TerminalBlock *blocks, const T *inv, const T *r, T *x) {
    const TerminalBlock tb = blocks[blockIdx.x];
    for (int p = static_cast<int>(threadIdx.x); p < tb.n; p += static_cast<int>(blockDim.x)) {
        const T *row = inv + tb.inv_offset + static_cast<std::int64_t>(p) * tb.n;
        T e = T(0);
        for (int q = 0; q < tb.n; ++q) {
            e += row[q] * r[tb.begin + q];
        }
        x[tb.begin + p] += e;
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
    const int k = find_sector_of(sectors, n_sectors, i);
    const SectorDesc &sec = sectors[k];
    if (i < 0 || i >= sec.begin + sec.size) {
        return;
    }
    std::int64_t rank[kMaxSpecies];
    split_local(sec, S, i - sec.begin, rank);
    int u[64];
    for (int s = 0; s < S; ++s) {
        unrank_species(B, rank[s], sec.total[s], V, u);
        for (int p = 0; p < sec.total[s]; ++p) {
            out[static_cast<std::int64_t>(V - 1 - u[p]) * S + s] += 1;
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
    int u[64];
    for (int s = 0; s < S; ++s) {
        if (totals[s] > 64) {
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
        local += rank_species(B, u, n) * sec.stride[s];
    }
    index[t] = sec.begin + local;
}

} // namespace

template <typename T>
cudaError_t launch_rows(RowMode mode, int mol_cap, const RowParams<T> &p, cudaStream_t stream) {
    switch (mol_cap) {
    case 4:
        return launch_mode<T, 4>(mode, p, stream);
    case 16:
        return launch_mode<T, 16>(mode, p, stream);
    case 64:
        return launch_mode<T, 64>(mode, p, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_rows<double>(RowMode, int, const RowParams<double> &, cudaStream_t);
template cudaError_t launch_rows<float>(RowMode, int, const RowParams<float> &, cudaStream_t);

template <typename T>
cudaError_t launch_terminal(const TerminalBlock *blocks, int n_blocks, const T *inv, const T *r,
                            T *x, cudaStream_t stream) {
    if (n_blocks == 0) {
        return cudaSuccess;
    }
    terminal_kernel<T><<<n_blocks, 128, 0, stream>>>(blocks, inv, r, x);
    return cudaGetLastError();
}

template cudaError_t launch_terminal<double>(const TerminalBlock *, int, const double *,
                                             const double *, double *, cudaStream_t);
template cudaError_t launch_terminal<float>(const TerminalBlock *, int, const float *,
                                            const float *, float *, cudaStream_t);

cudaError_t launch_unrank(const BinomTable &B, const SectorDesc *sectors, int n_sectors, int S,
                          int V, const std::int64_t *index, std::int64_t count, int *states,
                          cudaStream_t stream) {
    if (count == 0) {
        return cudaSuccess;
    }
    const int threads = 128;
    const auto blocks = static_cast<unsigned>((count + threads - 1) / threads);
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
    rank_kernel<<<blocks, threads, 0, stream>>>(B, sectors, n_sectors, max_totals, is_box, S, V,
                                                states, count, index);
    return cudaGetLastError();
}

} // namespace mkb
