// sm_100a Krylov kernels. All are HBM-bound streaming passes over the Arnoldi basis.
#include "krylov.cuh"
#include "launch_count.hpp"

#include <cmath>

namespace mkb {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

// reduce KMAX per-thread accumulators over the block; write partials[k * gridDim.x + block]
template <int KMAX>
__device__ __forceinline__ void block_partials(double (&acc)[KMAX], int K, double *partials) {
    __shared__ double red[kDotThreads / 32][KMAX];
    const int warp = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        if (k < K) {
            const double v = warp_sum(acc[k]);
            if (lane == 0) {
                red[warp][k] = v;
            }
        }
    }
    __syncthreads();
    for (int k = static_cast<int>(threadIdx.x); k < K; k += blockDim.x) {
        double s = 0.0;
        for (int wi = 0; wi < kDotThreads / 32; ++wi) {
            s += red[wi][k];
        }
        partials[static_cast<std::int64_t>(k) * gridDim.x + blockIdx.x] = s;
    }
}

// Blocks per SM the register budget is sized for (the tightest bounds that compile without
// spilling). The update-then-dots pass holds the loaded basis values and the accumulators at
// once; left unbounded, KMAX 16 takes 145 registers and one block per SM.
template <int KMAX, int MODE>
constexpr int cgs_min_blocks() {
    if constexpr (MODE == 4) {
        return cgs_min_blocks<KMAX, 0>();
    } else if constexpr (MODE == 5) {
        return cgs_min_blocks<KMAX, 1>();
    } else if constexpr (MODE == 1) {
        return KMAX >= 32 ? 1 : (KMAX >= 16 ? 2 : (KMAX >= 8 ? 3 : 4));
    } else if constexpr (MODE == 2) {
        return KMAX >= 16 ? 2 : 4;
    } else {
        return KMAX >= 32 ? 1 : (KMAX >= 16 ? (MODE == 0 ? 3 : 2) : 4);
    }
}

// mode 0: dots; mode 1: update then dots; mode 2: update then norm^2; mode 3: update only;
// modes 4 and 5: modes 0 and 1 with <w, w> after the K dots (entry K). A block returns at once
// when skip is set (the selective re-orthogonalisation's second pass, not needed).
// Each element's K basis values are loaded first (all in flight at once), then used. The update
// coefficients sit in shared memory (a broadcast read per use), which leaves the registers to
// the loaded values and the accumulators.
// Column blockIdx.y of a batch (ColumnBatch) sits at V + col * y, w + col * y,
// coef + coef_stride * y and partials + part_stride * y; columns whose mask bit is clear skip.
template <int KMAX, int MODE>
__global__ void __launch_bounds__(kDotThreads, (cgs_min_blocks<KMAX, MODE>()))
    cgs_kernel(const double *__restrict__ V, std::int64_t ld, int K, double *__restrict__ w,
               std::int64_t n, const double *__restrict__ coef, double *__restrict__ partials,
               std::int64_t col, std::int64_t coef_stride, std::int64_t part_stride,
               unsigned mask, const int *skip = nullptr) {
    if (!((mask >> blockIdx.y) & 1U) || (skip && *skip)) {
        return;
    }
    constexpr bool kNorm = MODE == 4 || MODE == 5;
    constexpr bool kDots = MODE == 0 || MODE == 1 || kNorm;
    constexpr bool kUpdate = MODE == 1 || MODE == 2 || MODE == 3 || MODE == 5;
    V += col * blockIdx.y;
    w += col * blockIdx.y;
    if (coef) {
        coef += coef_stride * blockIdx.y;
    }
    partials += part_stride * blockIdx.y;
    __shared__ double c[KMAX];
    if constexpr (kUpdate) {
        if (static_cast<int>(threadIdx.x) < KMAX) {
            c[threadIdx.x] = static_cast<int>(threadIdx.x) < K ? coef[threadIdx.x] : 0.0;
        }
        __syncthreads();
    }
    double acc[KMAX + 1];
#pragma unroll
    for (int k = 0; k <= KMAX; ++k) {
        acc[k] = 0.0;
    }
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        double v[KMAX];
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
            v[k] = k < K ? __ldcs(V + k * ld + i) : 0.0;
        }
        double wi = w[i];
        if constexpr (kUpdate) {
#pragma unroll
            for (int k = 0; k < KMAX; ++k) {
                wi -= c[k] * v[k];
            }
            w[i] = wi;
        }
        if constexpr (MODE == 2) {
            acc[0] += wi * wi;
        } else if constexpr (kDots) {
#pragma unroll
            for (int k = 0; k < KMAX; ++k) {
                acc[k] += v[k] * wi;
            }
            if constexpr (kNorm) {
                acc[KMAX] += wi * wi;
            }
        }
    }
    if constexpr (kNorm) {
        // the norm goes to entry K: move it down from the spare accumulator
        double tmp[KMAX + 1];
#pragma unroll
        for (int k = 0; k <= KMAX; ++k) {
            tmp[k] = k < K ? acc[k] : (k == K ? acc[KMAX] : 0.0);
        }
        block_partials<KMAX + 1>(tmp, K + 1, partials);
    } else if constexpr (MODE != 3) {
        block_partials<KMAX + 1>(acc, MODE == 2 ? 1 : K, partials);
    }
}

// out[k] = sum_b partials[k * nb + b], one warp per k, fixed order; block y serves column y of
// a batch (partials + part_stride * y, out + out_stride * y)
__global__ void finalize_kernel(const double *partials, int nb, int K, double *out,
                                std::int64_t part_stride, std::int64_t out_stride, unsigned mask,
                                const int *skip = nullptr) {
    if (!((mask >> blockIdx.x) & 1U) || (skip && *skip)) {
        return;
    }
    partials += part_stride * blockIdx.x;
    out += out_stride * blockIdx.x;
    const int warp = static_cast<int>(threadIdx.x) >> 5, lane = static_cast<int>(threadIdx.x) & 31;
    for (int k = warp; k < K; k += blockDim.x >> 5) {
        double s = 0.0;
        for (int b = lane; b < nb; b += 32) {
            s += partials[static_cast<std::int64_t>(k) * nb + b];
        }
        s = warp_sum(s);
        if (lane == 0) {
            out[k] = s;
        }
    }
}

template <int KMAX, int MODE>
cudaError_t launch_cgs(const double *V, std::int64_t ld, int K, double *w, std::int64_t n,
                       const double *coef, double *partials, double *out, cudaStream_t stream,
                       const int *skip = nullptr) {
    count_launches(MODE != 3 ? 2 : 1);
    cgs_kernel<KMAX, MODE><<<kDotBlocks, kDotThreads, 0, stream>>>(V, ld, K, w, n, coef, partials,
                                                                   0, 0, 0, 1U, skip);
    if (MODE != 3) {
        const int outs = MODE == 2 ? 1 : (MODE == 4 || MODE == 5 ? K + 1 : K);
        finalize_kernel<<<1, 1024, 0, stream>>>(partials, kDotBlocks, outs, out, 0, 0, 1U, skip);
    }
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_cgs_k(const double *V, std::int64_t ld, int K, double *w, std::int64_t n,
                         const double *coef, double *partials, double *out, cudaStream_t stream,
                         const int *skip = nullptr) {
    if (K <= 4) {
        return launch_cgs<4, MODE>(V, ld, K, w, n, coef, partials, out, stream, skip);
    }
    if (K <= 8) {
        return launch_cgs<8, MODE>(V, ld, K, w, n, coef, partials, out, stream, skip);
    }
    if (K <= 16) {
        return launch_cgs<16, MODE>(V, ld, K, w, n, coef, partials, out, stream, skip);
    }
    return launch_cgs<32, MODE>(V, ld, K, w, n, coef, partials, out, stream, skip);
}

// DGKS: after the first pass, w' = w - V h1; a second pass is needed only when
// ||w'||^2 < ||w||^2 / 2. Otherwise h2 = 0, <w', w'> is the norm, and the second pass's
// kernels return at once.
__global__ void dgks_kernel(const double *h1, double *h2, int K, double *hn, int *skip) {
    const bool enough = h2[K] >= 0.5 * h1[K];
    *skip = enough ? 1 : 0;
    if (enough) {
        *hn = h2[K];
        for (int k = 0; k < K; ++k) {
            h2[k] = 0.0;
        }
    }
}

// one CGS pass for every selected column of a batch: grid (kDotBlocks, nb), then nb finalizes
template <int KMAX, int MODE>
void launch_cgs_batch(const ColumnBatch &b, int K, const double *coef, double *out,
                      cudaStream_t stream) {
    const std::int64_t part = static_cast<std::int64_t>(kDotBlocks) * kMaxFusedBasis;
    count_launches(2);
    cgs_kernel<KMAX, MODE><<<dim3(kDotBlocks, b.nb), kDotThreads, 0, stream>>>(
        b.V, b.vstride, K, b.w, b.n, coef, b.partials, b.col, b.small, part, b.mask);
    finalize_kernel<<<b.nb, 1024, 0, stream>>>(b.partials, kDotBlocks, MODE == 2 ? 1 : K, out,
                                               part, b.small, b.mask);
}

template <int MODE>
void launch_cgs_batch_k(const ColumnBatch &b, int K, const double *coef, double *out,
                        cudaStream_t stream) {
    if (K <= 4) {
        launch_cgs_batch<4, MODE>(b, K, coef, out, stream);
    } else if (K <= 8) {
        launch_cgs_batch<8, MODE>(b, K, coef, out, stream);
    } else if (K <= 16) {
        launch_cgs_batch<16, MODE>(b, K, coef, out, stream);
    } else {
        launch_cgs_batch<32, MODE>(b, K, coef, out, stream);
    }
}

// y = x * (*scale); block row y of the grid serves column y of a batch
__global__ void scale_copy_batch_kernel(const double *x, const double *scale, double *y,
                                        std::int64_t n, std::int64_t col, std::int64_t small,
                                        unsigned mask) {
    if (!((mask >> blockIdx.y) & 1U)) {
        return;
    }
    x += col * blockIdx.y;
    y += col * blockIdx.y;
    const double a = scale[small * blockIdx.y];
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        y[i] = x[i] * a;
    }
}

__global__ void scale_copy_kernel(const double *x, const double *scale, double *y, std::int64_t n) {
    const double a = *scale;
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        y[i] = x[i] * a;
    }
}

template <bool ACCUMULATE>
__global__ void multi_axpy_kernel(const double *V, std::int64_t ld, int K, const double *coef,
                                  double *y, std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        double s = ACCUMULATE ? y[i] : 0.0;
        for (int k = 0; k < K; ++k) {
            s += coef[k] * V[k * ld + i];
        }
        y[i] = s;
    }
}

__global__ void axpy_kernel(double a, const double *x, double *y, std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        y[i] += a * x[i];
    }
}

template <typename A, typename B>
__global__ void convert_kernel(const A *x, B *y, std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        y[i] = static_cast<B>(x[i]);
    }
}

unsigned stream_blocks(std::int64_t n) {
    const std::int64_t want = (n + 255) / 256;
    return static_cast<unsigned>(want < 148 * 8 ? (want > 0 ? want : 1) : 148 * 8);
}

__global__ void arnoldi_start_kernel(ArnoldiState s) {
    const double norm = sqrt(*s.beta);
    for (int i = 0; i <= s.m; ++i) {
        s.g[i] = 0.0;
    }
    s.g[0] = norm;
    *s.beta = norm > 0.0 ? 1.0 / norm : 0.0;
    s.report[0] = norm;
    s.report[1] = norm;
    s.report[2] = 0.0;
}

__device__ void arnoldi_column_step(const ArnoldiState &s, int j) {
    const int ld = s.m + 1;
    double *col = s.H + static_cast<std::int64_t>(j) * ld;
    for (int i = 0; i <= j; ++i) {
        col[i] = s.h1[i] + s.h2[i];
    }
    const double hn = sqrt(*s.hn);
    col[j + 1] = hn;
    for (int i = 0; i < j; ++i) {
        const double a = col[i], c = col[i + 1];
        col[i] = s.cs[i] * a + s.sn[i] * c;
        col[i + 1] = -s.sn[i] * a + s.cs[i] * c;
    }
    const double a = col[j], c = col[j + 1];
    const double denom = hypot(a, c);
    s.cs[j] = denom > 0.0 ? a / denom : 1.0;
    s.sn[j] = denom > 0.0 ? c / denom : 0.0;
    col[j] = denom;
    col[j + 1] = 0.0;
    s.g[j + 1] = -s.sn[j] * s.g[j];
    s.g[j] = s.cs[j] * s.g[j];
    *s.inv_hn = hn > 0.0 ? 1.0 / hn : 0.0;
    s.report[0] = fabs(s.g[j + 1]);
    s.report[1] = hn;
    s.report[2] = (hn > 0.0 && isfinite(hn)) ? 0.0 : 1.0;
}

__global__ void arnoldi_column_kernel(ArnoldiState s, int j) { arnoldi_column_step(s, j); }

// block c: the Givens column of batch column c, its report also copied to reports + 4 c
__global__ void arnoldi_column_batch_kernel(ArnoldiState s0, std::int64_t small, unsigned mask,
                                            int j, double *reports) {
    const int c = static_cast<int>(blockIdx.x);
    if (!((mask >> c) & 1U)) {
        return;
    }
    ArnoldiState s = s0;
    const std::int64_t off = small * c;
    s.H += off;
    s.cs += off;
    s.sn += off;
    s.g += off;
    s.y += off;
    s.h1 += off;
    s.h2 += off;
    s.hn += off;
    s.inv_hn += off;
    s.beta += off;
    s.report += off;
    arnoldi_column_step(s, j);
    for (int k = 0; k < 4; ++k) {
        reports[4 * c + k] = s.report[k];
    }
}

__global__ void arnoldi_solve_kernel(ArnoldiState s, int k) {
    const int ld = s.m + 1;
    for (int i = k - 1; i >= 0; --i) {
        double v = s.g[i];
        for (int t = i + 1; t < k; ++t) {
            v -= s.H[static_cast<std::int64_t>(t) * ld + i] * s.y[t];
        }
        s.y[i] = v / s.H[static_cast<std::int64_t>(i) * ld + i];
    }
}

} // namespace

cudaError_t cgs_dgks(const double *V, std::int64_t ld, int K, double *w, std::int64_t n,
                     double *partials, double *h1, double *h2, double *hn, int *skip,
                     cudaStream_t stream) {
    if (K < 1 || K >= kMaxFusedBasis) {
        return cudaErrorInvalidValue;
    }
    cudaError_t e = launch_cgs_k<4>(V, ld, K, w, n, nullptr, partials, h1, stream);
    if (e == cudaSuccess) {
        e = launch_cgs_k<5>(V, ld, K, w, n, h1, partials, h2, stream);
    }
    if (e == cudaSuccess) {
        count_launches(1);
        dgks_kernel<<<1, 1, 0, stream>>>(h1, h2, K, hn, skip);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        e = launch_cgs_k<2>(V, ld, K, w, n, h2, partials, hn, stream, skip);
    }
    return e;
}

cudaError_t cgs_pass(int mode, const double *V, std::int64_t ld, int K, double *w, std::int64_t n,
                     const double *coef, double *partials, double *out, cudaStream_t stream) {
    if (K < 1 || K > kMaxFusedBasis) {
        return cudaErrorInvalidValue;
    }
    switch (mode) {
    case 0:
        return launch_cgs_k<0>(V, ld, K, w, n, coef, partials, out, stream);
    case 1:
        return launch_cgs_k<1>(V, ld, K, w, n, coef, partials, out, stream);
    case 2:
        return launch_cgs_k<2>(V, ld, K, w, n, coef, partials, out, stream);
    case 3:
        return launch_cgs_k<3>(V, ld, K, w, n, coef, partials, out, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

cudaError_t cgs_step_batch(const ColumnBatch &b, int j, bool next, cudaStream_t stream) {
    const int K = j + 1;
    if (K < 1 || K > kMaxFusedBasis || b.nb < 1 || b.nb > 32) {
        return cudaErrorInvalidValue;
    }
    const ArnoldiState &s = b.st;
    launch_cgs_batch_k<0>(b, K, nullptr, s.h1, stream);
    launch_cgs_batch_k<1>(b, K, s.h1, s.h2, stream);
    launch_cgs_batch_k<2>(b, K, s.h2, s.hn, stream);
    count_launches(1);
    arnoldi_column_batch_kernel<<<b.nb, 1, 0, stream>>>(s, b.small, b.mask, j, b.reports);
    if (next) {
        count_launches(1);
        scale_copy_batch_kernel<<<dim3(stream_blocks(b.n), b.nb), 256, 0, stream>>>(
            b.w, s.inv_hn, b.V + static_cast<std::int64_t>(j + 1) * b.vstride, b.n, b.col,
            b.small, b.mask);
    }
    return cudaGetLastError();
}

cudaError_t dot(const double *a, const double *b, std::int64_t n, double *partials, double *out,
                cudaStream_t stream) {
    // <a, b> as a one-vector "basis" pass
    return launch_cgs<4, 0>(a, n, 1, const_cast<double *>(b), n, nullptr, partials, out, stream);
}

cudaError_t scale_copy(const double *x, const double *scale, double *y, std::int64_t n,
                       cudaStream_t stream) {
    count_launches(1);
    scale_copy_kernel<<<stream_blocks(n), 256, 0, stream>>>(x, scale, y, n);
    return cudaGetLastError();
}

cudaError_t multi_axpy(const double *V, std::int64_t ld, int K, const double *coef, double *y,
                       std::int64_t n, cudaStream_t stream) {
    count_launches(1);
    multi_axpy_kernel<true><<<stream_blocks(n), 256, 0, stream>>>(V, ld, K, coef, y, n);
    return cudaGetLastError();
}

cudaError_t multi_combine(const double *V, std::int64_t ld, int K, const double *coef, double *y,
                          std::int64_t n, cudaStream_t stream) {
    count_launches(1);
    multi_axpy_kernel<false><<<stream_blocks(n), 256, 0, stream>>>(V, ld, K, coef, y, n);
    return cudaGetLastError();
}

cudaError_t axpy(double a, const double *x, double *y, std::int64_t n, cudaStream_t stream) {
    count_launches(1);
    axpy_kernel<<<stream_blocks(n), 256, 0, stream>>>(a, x, y, n);
    return cudaGetLastError();
}

template <typename A, typename B>
cudaError_t convert(const A *x, B *y, std::int64_t n, cudaStream_t stream) {
    count_launches(1);
    convert_kernel<A, B><<<stream_blocks(n), 256, 0, stream>>>(x, y, n);
    return cudaGetLastError();
}
template cudaError_t convert<double, float>(const double *, float *, std::int64_t, cudaStream_t);
template cudaError_t convert<float, double>(const float *, double *, std::int64_t, cudaStream_t);

cudaError_t arnoldi_start(const ArnoldiState &s, cudaStream_t stream) {
    count_launches(1);
    arnoldi_start_kernel<<<1, 1, 0, stream>>>(s);
    return cudaGetLastError();
}

cudaError_t arnoldi_column(const ArnoldiState &s, int j, cudaStream_t stream) {
    count_launches(1);
    arnoldi_column_kernel<<<1, 1, 0, stream>>>(s, j);
    return cudaGetLastError();
}

cudaError_t arnoldi_solve(const ArnoldiState &s, int k, cudaStream_t stream) {
    count_launches(1);
    arnoldi_solve_kernel<<<1, 1, 0, stream>>>(s, k);
    return cudaGetLastError();
}

} // namespace mkb
