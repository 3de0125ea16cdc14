// Diagonal, ILU(0) and host-callback preconditioners of gmres() (precond.cuh).
#include "launch_count.hpp"
#include "precond.cuh"

#include <algorithm>
#include <climits>
#include <cmath>

namespace mkb {
namespace {

constexpr int kThreads = 256;
constexpr int kNarrowThreads = 1024;

__global__ void scale_kernel(const double *__restrict__ d, const double *__restrict__ v,
                             double *__restrict__ z, std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        z[i] = d[i] * v[i];
    }
}

// the factors in A's pattern; val is rewritten in place by the factorisation
struct IluView {
    const std::int64_t *ptr;
    const std::int64_t *diag;
    const int *col;
    double *val;
};

enum Sweep : int { kFactor = 0, kLower = 1, kUpper = 2 };

// IKJ: row i's entries left of the diagonal in ascending column order, each divided by its
// pivot and then eliminated from the rest of row i through row k's U part (a merge of two
// ascending column lists)
__device__ void factor_row(const IluView a, int i) {
    const std::int64_t end = a.ptr[i + 1], di = a.diag[i];
    for (std::int64_t p = a.ptr[i]; p < di; ++p) {
        const int k = a.col[p];
        const std::int64_t dk = a.diag[k], ek = a.ptr[k + 1];
        const double l = a.val[p] / a.val[dk];
        a.val[p] = l;
        std::int64_t q = dk + 1, r = p + 1;
        while (q < ek && r < end) {
            const int cq = a.col[q], cr = a.col[r];
            if (cq == cr) {
                a.val[r] = fma(-l, a.val[q], a.val[r]);
                ++q;
                ++r;
            } else if (cq < cr) {
                ++q;
            } else {
                ++r;
            }
        }
    }
}

// y_i = v_i - sum_{j < i} l_ij y_j
__device__ void lower_row(const IluView a, int i, const double *v, double *y) {
    double s = v[i];
    for (std::int64_t p = a.ptr[i], e = a.diag[i]; p < e; ++p) {
        s = fma(-a.val[p], y[a.col[p]], s);
    }
    y[i] = s;
}

// z_i = (y_i - sum_{j > i} u_ij z_j) / u_ii
__device__ void upper_row(const IluView a, int i, const double *y, double *z) {
    const std::int64_t di = a.diag[i];
    double s = y[i];
    for (std::int64_t p = di + 1, e = a.ptr[i + 1]; p < e; ++p) {
        s = fma(-a.val[p], z[a.col[p]], s);
    }
    z[i] = s / a.val[di];
}

template <int SWEEP>
__device__ __forceinline__ void visit(const IluView a, int i, const double *in, double *out) {
    if constexpr (SWEEP == kFactor) {
        factor_row(a, i);
    } else if constexpr (SWEEP == kLower) {
        lower_row(a, i, in, out);
    } else {
        upper_row(a, i, in, out);
    }
}

// one level over a grid
template <int SWEEP>
__global__ void __launch_bounds__(kThreads)
    wide_level_kernel(const IluView a, const int *__restrict__ order,
                      const std::int64_t *__restrict__ level_ptr, std::int64_t l,
                      const double *in, double *out) {
    const std::int64_t b = level_ptr[l], e = level_ptr[l + 1];
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t t = b + blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         t < e; t += stride) {
        visit<SWEEP>(a, order[t], in, out);
    }
}

// one level over a grid, a warp per row: the lanes stride the row's entries and the partial
// sums meet by shuffles (triangular solves only)
template <int SWEEP>
__global__ void __launch_bounds__(kThreads)
    warp_level_kernel(const IluView a, const int *__restrict__ order,
                      const std::int64_t *__restrict__ level_ptr, std::int64_t l,
                      const double *in, double *out) {
    static_assert(SWEEP == kLower || SWEEP == kUpper, "solves only");
    const std::int64_t b = level_ptr[l], e = level_ptr[l + 1];
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const std::int64_t warps = static_cast<std::int64_t>(gridDim.x) * (blockDim.x / 32);
    for (std::int64_t t = b + (blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x) / 32;
         t < e; t += warps) {
        const int i = order[t];
        const std::int64_t di = a.diag[i];
        const std::int64_t p0 = SWEEP == kLower ? a.ptr[i] : di + 1;
        const std::int64_t p1 = SWEEP == kLower ? di : a.ptr[i + 1];
        double s = 0.0;
        for (std::int64_t p = p0 + lane; p < p1; p += 32) {
            s = fma(a.val[p], out[a.col[p]], s);
        }
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffU, s, o);
        }
        if (lane == 0) {
            out[i] = SWEEP == kLower ? in[i] - s : (in[i] - s) / a.val[di];
        }
    }
}

// levels [l0, l1) in one block, a barrier after each so the next level sees its rows
template <int SWEEP>
__global__ void __launch_bounds__(kNarrowThreads)
    narrow_levels_kernel(const IluView a, const int *__restrict__ order,
                         const std::int64_t *__restrict__ level_ptr, std::int64_t l0,
                         std::int64_t l1, const double *in, double *out) {
    for (std::int64_t l = l0; l < l1; ++l) {
        const std::int64_t e = level_ptr[l + 1];
        for (std::int64_t t = level_ptr[l] + threadIdx.x; t < e; t += kNarrowThreads) {
            visit<SWEEP>(a, order[t], in, out);
        }
        __syncthreads();
    }
}

__global__ void pivot_check_kernel(const double *__restrict__ val,
                                   const std::int64_t *__restrict__ diag, std::int64_t n,
                                   int *bad) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        const double d = val[diag[i]];
        if (!isfinite(d) || d == 0.0) {
            *bad = 1; // every writer stores the same value
        }
    }
}

unsigned grid_for(std::int64_t work) {
    const std::int64_t blocks = (work + kThreads - 1) / kThreads;
    return static_cast<unsigned>(std::clamp<std::int64_t>(blocks, 1, 148 * 16));
}

// levels of the lower (dependencies j < i) or upper (j > i) sweep, rows grouped by level
void build_schedule(std::int64_t n, const std::vector<std::int64_t> &ptr,
                    const std::vector<int> &col, const std::vector<std::int64_t> &diag,
                    bool lower_sweep, LevelSchedule &s) {
    std::vector<std::int64_t> lev(static_cast<std::size_t>(n), 0);
    std::int64_t depth = 0;
    auto level_of = [&](std::int64_t i, std::int64_t b, std::int64_t e) {
        std::int64_t m = -1;
        for (std::int64_t p = b; p < e; ++p) {
            m = std::max(m, lev[col[p]]);
        }
        lev[i] = m + 1;
        depth = std::max(depth, m + 2);
    };
    if (lower_sweep) {
        for (std::int64_t i = 0; i < n; ++i) {
            level_of(i, ptr[i], diag[i]);
        }
    } else {
        for (std::int64_t i = n - 1; i >= 0; --i) {
            level_of(i, diag[i] + 1, ptr[i + 1]);
        }
    }
    s.h_level_ptr.assign(static_cast<std::size_t>(depth) + 1, 0);
    for (std::int64_t i = 0; i < n; ++i) {
        ++s.h_level_ptr[lev[i] + 1];
    }
    for (std::int64_t l = 0; l < depth; ++l) {
        s.h_level_ptr[l + 1] += s.h_level_ptr[l];
    }
    std::vector<int> order(static_cast<std::size_t>(n));
    std::vector<std::int64_t> fill(s.h_level_ptr.begin(), s.h_level_ptr.end() - 1);
    std::vector<std::int64_t> work(static_cast<std::size_t>(depth), 0), longest(work);
    for (std::int64_t i = 0; i < n; ++i) {
        order[fill[lev[i]]++] = static_cast<int>(i);
        const std::int64_t len = lower_sweep ? diag[i] - ptr[i] : ptr[i + 1] - diag[i] - 1;
        work[lev[i]] += len + 1;
        longest[lev[i]] = std::max(longest[lev[i]], len);
    }
    s.order.upload(order);
    s.level_ptr.upload(s.h_level_ptr);
    s.segments.clear();
    for (std::int64_t l = 0; l < depth; ++l) {
        const std::int64_t rows = s.h_level_ptr[l + 1] - s.h_level_ptr[l];
        if (rows > Ilu0Preconditioner::kNarrowRows || work[l] > Ilu0Preconditioner::kNarrowWork) {
            s.segments.push_back({l, l + 1, rows, true,
                                  longest[l] > Ilu0Preconditioner::kWarpRowLength});
        } else if (!s.segments.empty() && !s.segments.back().wide) {
            s.segments.back().l1 = l + 1;
            s.segments.back().rows += rows;
        } else {
            s.segments.push_back({l, l + 1, rows, false, false});
        }
    }
}

template <int SWEEP>
void run_schedule(const IluView a, const LevelSchedule &s, const double *in, double *out,
                  cudaStream_t stream) {
    for (const auto &g : s.segments) {
        if constexpr (SWEEP != kFactor) {
            if (g.warp) {
                warp_level_kernel<SWEEP><<<grid_for(32 * g.rows), kThreads, 0, stream>>>(
                    a, s.order.get(), s.level_ptr.get(), g.l0, in, out);
                continue;
            }
        }
        if (g.wide) {
            wide_level_kernel<SWEEP><<<grid_for(g.rows), kThreads, 0, stream>>>(
                a, s.order.get(), s.level_ptr.get(), g.l0, in, out);
        } else {
            narrow_levels_kernel<SWEEP><<<1, kNarrowThreads, 0, stream>>>(
                a, s.order.get(), s.level_ptr.get(), g.l0, g.l1, in, out);
        }
    }
    count_launches(s.segments.size());
    check_cuda(cudaGetLastError(), "ILU(0) sweep");
}

} // namespace

DiagonalPreconditioner::DiagonalPreconditioner(const double *inverse_diagonal_host, std::int64_t n_)
    : Preconditioner(n_) {
    if (n_ < 1 || !inverse_diagonal_host) {
        throw Error(kEInval, "jacobi preconditioner: empty inverse diagonal");
    }
    d.upload(std::vector<double>(inverse_diagonal_host, inverse_diagonal_host + n_));
}

void DiagonalPreconditioner::apply(const double *v, double *z, cudaStream_t stream) {
    scale_kernel<<<grid_for(n), kThreads, 0, stream>>>(d.get(), v, z, n);
    count_launches(1);
    check_cuda(cudaGetLastError(), "jacobi preconditioner");
}

Ilu0Preconditioner::Ilu0Preconditioner(std::int64_t n_, const std::int64_t *row_ptr,
                                       const std::int64_t *cols, const double *vals,
                                       cudaStream_t stream)
    : Preconditioner(n_) {
    if (n_ < 1 || n_ >= INT_MAX || !row_ptr || !cols || !vals) {
        throw Error(kEInval, "ilu0 preconditioner: bad matrix");
    }
    const std::int64_t nnz = row_ptr[n_];
    if (row_ptr[0] != 0 || nnz < n_) {
        throw Error(kEInval, "ilu0 preconditioner: bad row pointers");
    }
    std::vector<std::int64_t> hptr(row_ptr, row_ptr + n_ + 1), hdiag(static_cast<std::size_t>(n_));
    std::vector<int> hcol(static_cast<std::size_t>(nnz));
    for (std::int64_t i = 0; i < n_; ++i) {
        if (hptr[i + 1] < hptr[i] || hptr[i + 1] > nnz) {
            throw Error(kEInval, "ilu0 preconditioner: bad row pointers");
        }
        hdiag[i] = -1;
        for (std::int64_t p = hptr[i]; p < hptr[i + 1]; ++p) {
            const std::int64_t c = cols[p];
            if (c < 0 || c >= n_ || (p > hptr[i] && c <= cols[p - 1])) {
                throw Error(kEInval, "ilu0 preconditioner: columns must be in range and strictly "
                                     "ascending within each row");
            }
            hcol[p] = static_cast<int>(c);
            if (c == i) {
                hdiag[i] = p;
            }
        }
        if (hdiag[i] < 0) {
            throw Error(kEInval, "ilu0 preconditioner: a row has no diagonal entry");
        }
    }
    ptr.upload(hptr);
    diag.upload(hdiag);
    col.upload(hcol);
    val.resize(static_cast<std::size_t>(nnz));
    check_cuda(cudaMemcpyAsync(val.get(), vals, static_cast<std::size_t>(nnz) * sizeof(double),
                               cudaMemcpyHostToDevice, stream),
               "upload");
    build_schedule(n_, hptr, hcol, hdiag, true, lower);
    build_schedule(n_, hptr, hcol, hdiag, false, upper);
    y.resize(static_cast<std::size_t>(n_));
    const IluView a{ptr.get(), diag.get(), col.get(), val.get()};
    run_schedule<kFactor>(a, lower, nullptr, nullptr, stream);
    DeviceArray<int> bad(1);
    check_cuda(cudaMemsetAsync(bad.get(), 0, sizeof(int), stream), "pivots");
    pivot_check_kernel<<<grid_for(n_), kThreads, 0, stream>>>(val.get(), diag.get(), n_, bad.get());
    count_launches(1);
    check_cuda(cudaGetLastError(), "pivots");
    int h_bad = 0;
    check_cuda(cudaMemcpyAsync(&h_bad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, stream),
               "pivots");
    check_cuda(cudaStreamSynchronize(stream), "sync");
    if (h_bad) {
        throw Error(kESingular, "ilu0 preconditioner: zero or non-finite pivot");
    }
}

void Ilu0Preconditioner::apply(const double *v, double *z, cudaStream_t stream) {
    const IluView a{ptr.get(), diag.get(), col.get(), val.get()};
    run_schedule<kLower>(a, lower, v, y.get(), stream);
    run_schedule<kUpper>(a, upper, y.get(), z, stream);
}

HostPreconditioner::HostPreconditioner(std::int64_t n_, Fn f, void *c)
    : Preconditioner(n_), fn(f), ctx(c) {
    if (n_ < 1 || !f) {
        throw Error(kEInval, "host preconditioner: null callback or empty size");
    }
    const std::size_t bytes = static_cast<std::size_t>(n_) * sizeof(double);
    check_cuda(cudaMallocHost(reinterpret_cast<void **>(&hv), bytes), "cudaMallocHost");
    if (cudaMallocHost(reinterpret_cast<void **>(&hz), bytes) != cudaSuccess) {
        cudaFreeHost(hv);
        throw Error(kENoMem, "cudaMallocHost failed");
    }
}

HostPreconditioner::~HostPreconditioner() {
    cudaFreeHost(hv);
    cudaFreeHost(hz);
}

void HostPreconditioner::apply(const double *v, double *z, cudaStream_t stream) {
    const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(double);
    check_cuda(cudaMemcpyAsync(hv, v, bytes, cudaMemcpyDeviceToHost, stream), "d2h");
    check_cuda(cudaStreamSynchronize(stream), "sync");
    if (fn(ctx, hv, hz, n) != 0) {
        throw Error(kEInval, "host preconditioner returned an error");
    }
    check_cuda(cudaMemcpyAsync(z, hz, bytes, cudaMemcpyHostToDevice, stream), "h2d");
    check_cuda(cudaStreamSynchronize(stream), "sync");
}

} // namespace mkb
