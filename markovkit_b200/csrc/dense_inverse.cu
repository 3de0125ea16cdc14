// Gauss-Jordan inverses of dense terminal blocks, on the host or, for large blocks, on the
// device with the same arithmetic (dense_inverse.cuh).
#include "dense_inverse.cuh"
#include "engine.hpp"
#include "launch_count.hpp"

#include <algorithm>
#include <cmath>

namespace mkb {
namespace {

constexpr int kPivotThreads = 1024;
constexpr int kElimThreads = 256;
// below this much work (sum of n^3) the host routine is as quick as the launches
constexpr double kDeviceWork = 1.6e7;

// one augmented block [A | I], row-major with 2 n columns at m_off; its pivot column at f_off
struct GjBlock {
    std::int64_t m_off = 0;
    std::int64_t f_off = 0;
    int n = 0;
    int pad = 0;
};

// step k of one block per CUDA block: the pivot row (the first row of largest |a_ik|, i >= k),
// the swap, the scaling of row k by its pivot, and a copy of column k for the elimination
__global__ void __launch_bounds__(kPivotThreads)
    gj_pivot_kernel(const GjBlock *__restrict__ blocks, double *M, double *f, int k, int *singular) {
    const GjBlock g = blocks[blockIdx.x];
    const int n = g.n;
    if (k >= n) {
        return;
    }
    const std::int64_t w = 2 * static_cast<std::int64_t>(n);
    double *m = M + g.m_off;
    const int tid = static_cast<int>(threadIdx.x);
    double best = -1.0;
    int at = n;
    for (int i = k + tid; i < n; i += kPivotThreads) {
        const double v = fabs(m[i * w + k]);
        if (v > best) {
            best = v;
            at = i;
        }
    }
    // larger magnitude wins; equal magnitudes go to the lower row, as in a sequential scan
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffU, best, o);
        const int oa = __shfl_down_sync(0xffffffffU, at, o);
        if (ob > best || (ob == best && oa < at)) {
            best = ob;
            at = oa;
        }
    }
    __shared__ double s_best[kPivotThreads / 32];
    __shared__ int s_at[kPivotThreads / 32];
    __shared__ int s_p;
    if ((tid & 31) == 0) {
        s_best[tid >> 5] = best;
        s_at[tid >> 5] = at;
    }
    __syncthreads();
    if (tid == 0) {
        double b = s_best[0];
        int a = s_at[0];
        for (int q = 1; q < kPivotThreads / 32; ++q) {
            if (s_best[q] > b || (s_best[q] == b && s_at[q] < a)) {
                b = s_best[q];
                a = s_at[q];
            }
        }
        s_p = a;
    }
    __syncthreads();
    const int p = s_p;
    if (p >= n || m[p * w + k] == 0.0) {
        if (tid == 0) {
            *singular = 1; // every writer stores the same value
        }
        return;
    }
    if (p != k) {
        for (std::int64_t j = tid; j < w; j += kPivotThreads) {
            const double t = m[k * w + j];
            m[k * w + j] = m[p * w + j];
            m[p * w + j] = t;
        }
    }
    __syncthreads();
    const double d = m[k * w + k];
    __syncthreads();
    for (std::int64_t j = tid; j < w; j += kPivotThreads) {
        m[k * w + j] = __ddiv_rn(m[k * w + j], d);
    }
    __syncthreads();
    for (int i = tid; i < n; i += kPivotThreads) {
        f[g.f_off + i] = m[i * w + k];
    }
}

// rows i != k: row_i -= f_i row_k over the columns that can change (k.. of A, all of the
// inverse); a rounded product, then a rounded difference
__global__ void __launch_bounds__(kElimThreads)
    gj_eliminate_kernel(const GjBlock *__restrict__ blocks, double *M, const double *__restrict__ f,
                        int k) {
    const GjBlock g = blocks[blockIdx.y];
    const int n = g.n;
    if (k >= n) {
        return;
    }
    const std::int64_t w = 2 * static_cast<std::int64_t>(n);
    const std::int64_t cw = w - k;
    const std::int64_t total = static_cast<std::int64_t>(n) * cw;
    double *m = M + g.m_off;
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t idx = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         idx < total; idx += stride) {
        const std::int64_t i = idx / cw;
        const std::int64_t j = k + idx % cw;
        if (i == k) {
            continue;
        }
        const double fi = f[g.f_off + i];
        if (fi == 0.0) {
            continue;
        }
        m[i * w + j] = __dsub_rn(m[i * w + j], __dmul_rn(fi, m[k * w + j]));
    }
}

} // namespace

// dense inverse by Gauss-Jordan with partial pivoting; false when singular
bool invert_dense(std::vector<double> &A, int n, std::vector<double> &inv) {
    inv.assign(static_cast<std::size_t>(n) * n, 0.0);
    for (int i = 0; i < n; ++i) {
        inv[static_cast<std::size_t>(i) * n + i] = 1.0;
    }
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i) {
            if (std::abs(A[static_cast<std::size_t>(i) * n + k]) >
                std::abs(A[static_cast<std::size_t>(p) * n + k])) {
                p = i;
            }
        }
        if (A[static_cast<std::size_t>(p) * n + k] == 0.0) {
            return false;
        }
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                std::swap(A[static_cast<std::size_t>(k) * n + j], A[static_cast<std::size_t>(p) * n + j]);
                std::swap(inv[static_cast<std::size_t>(k) * n + j],
                          inv[static_cast<std::size_t>(p) * n + j]);
            }
        }
        const double d = A[static_cast<std::size_t>(k) * n + k];
        for (int j = 0; j < n; ++j) {
            A[static_cast<std::size_t>(k) * n + j] /= d;
            inv[static_cast<std::size_t>(k) * n + j] /= d;
        }
        for (int i = 0; i < n; ++i) {
            if (i == k) {
                continue;
            }
            const double f = A[static_cast<std::size_t>(i) * n + k];
            if (f == 0.0) {
                continue;
            }
            for (int j = 0; j < n; ++j) {
                A[static_cast<std::size_t>(i) * n + j] -= f * A[static_cast<std::size_t>(k) * n + j];
                inv[static_cast<std::size_t>(i) * n + j] -= f * inv[static_cast<std::size_t>(k) * n + j];
            }
        }
    }
    return true;
}

bool invert_dense_blocks(std::vector<double> &A, const std::vector<std::int64_t> &offset,
                         const std::vector<int> &n, std::vector<double> &inv) {
    inv.assign(A.size(), 0.0);
    double work = 0.0;
    int nmax = 0;
    for (int b : n) {
        work += static_cast<double>(b) * b * b;
        nmax = std::max(nmax, b);
    }
    if (work < kDeviceWork) {
        std::vector<double> a, x;
        for (std::size_t b = 0; b < n.size(); ++b) {
            const std::size_t nn = static_cast<std::size_t>(n[b]) * n[b];
            a.assign(A.begin() + offset[b], A.begin() + offset[b] + static_cast<std::ptrdiff_t>(nn));
            if (!invert_dense(a, n[b], x)) {
                return false;
            }
            std::copy(x.begin(), x.end(), inv.begin() + offset[b]);
        }
        return true;
    }
    // [A | I] per block on the device
    std::vector<GjBlock> hb(n.size());
    std::int64_t m_total = 0, f_total = 0;
    for (std::size_t b = 0; b < n.size(); ++b) {
        hb[b].m_off = m_total;
        hb[b].f_off = f_total;
        hb[b].n = n[b];
        m_total += 2 * static_cast<std::int64_t>(n[b]) * n[b];
        f_total += n[b];
    }
    std::vector<double> aug(static_cast<std::size_t>(m_total), 0.0);
    for (std::size_t b = 0; b < n.size(); ++b) {
        const std::int64_t nb = n[b], w = 2 * nb;
        for (std::int64_t i = 0; i < nb; ++i) {
            std::copy(A.begin() + offset[b] + i * nb, A.begin() + offset[b] + (i + 1) * nb,
                      aug.begin() + hb[b].m_off + i * w);
            aug[hb[b].m_off + i * w + nb + i] = 1.0;
        }
    }
    DeviceArray<GjBlock> d_blocks;
    d_blocks.upload(hb);
    DeviceArray<double> M, f(static_cast<std::size_t>(f_total));
    M.upload(aug);
    DeviceArray<int> singular(1);
    check_cuda(cudaMemset(singular.get(), 0, sizeof(int)), "memset");
    const auto nblk = static_cast<unsigned>(n.size());
    const std::int64_t widest = 2 * static_cast<std::int64_t>(nmax) * nmax;
    const unsigned gx = static_cast<unsigned>(std::clamp<std::int64_t>(
        (widest + kElimThreads - 1) / kElimThreads, 1, 148 * 8));
    for (int k = 0; k < nmax; ++k) {
        gj_pivot_kernel<<<nblk, kPivotThreads>>>(d_blocks.get(), M.get(), f.get(), k, singular.get());
        gj_eliminate_kernel<<<dim3(gx, nblk), kElimThreads>>>(d_blocks.get(), M.get(), f.get(), k);
    }
    count_launches(2 * static_cast<std::uint64_t>(nmax));
    check_cuda(cudaGetLastError(), "dense inverse");
    int h_singular = 0;
    check_cuda(cudaMemcpy(&h_singular, singular.get(), sizeof(int), cudaMemcpyDeviceToHost), "d2h");
    if (h_singular) {
        return false;
    }
    check_cuda(cudaMemcpy(aug.data(), M.get(), aug.size() * sizeof(double), cudaMemcpyDeviceToHost),
               "d2h");
    for (std::size_t b = 0; b < n.size(); ++b) {
        const std::int64_t nb = n[b], w = 2 * nb;
        for (std::int64_t i = 0; i < nb; ++i) {
            std::copy(aug.begin() + hb[b].m_off + i * w + nb, aug.begin() + hb[b].m_off + i * w + w,
                      inv.begin() + offset[b] + i * nb);
        }
    }
    return true;
}

} // namespace mkb
