// Fixed-order multigrid transfers (transfer.cuh).
#include "launch_count.hpp"
#include "transfer.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <type_traits>

namespace mkb {
namespace {

constexpr int kThreads = 256;

unsigned grid_for(std::int64_t n) {
    return static_cast<unsigned>(std::max<std::int64_t>(1, std::min<std::int64_t>((n + kThreads - 1) / kThreads, 148 * 16)));
}

__global__ void iota_kernel(int *v, std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        v[i] = static_cast<int>(i);
    }
}

// begin[c] = first position of key c in the sorted keys (lower bound), c = 0 .. n_coarse
__global__ void bounds_kernel(const int *keys, std::int64_t n_fine, std::int64_t n_coarse,
                              int *begin) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t c = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         c <= n_coarse; c += stride) {
        std::int64_t lo = 0, hi = n_fine;
        while (lo < hi) {
            const std::int64_t mid = (lo + hi) >> 1;
            if (keys[mid] < c) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        begin[c] = static_cast<int>(lo);
    }
}

template <typename T>
__global__ void restrict_kernel(const int *begin, const int *children, std::int64_t n_coarse,
                                const T *fine, std::int64_t ldf, T *coarse, std::int64_t ldc,
                                int nb) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t c = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         c < n_coarse; c += stride) {
        const int k0 = begin[c], k1 = begin[c + 1];
        for (int col = 0; col < nb; ++col) {
            const T *f = fine + col * ldf;
            T acc = T(0);
            for (int k = k0; k < k1; ++k) {
                acc += f[__ldg(children + k)];
            }
            coarse[c + col * ldc] = acc;
        }
    }
}

// the interleaved FP32 batch: four lanes per entry, one 16-byte load per child
__global__ void restrict_lanes_kernel(const int *begin, const int *children, std::int64_t n_coarse,
                                      const float *fine, float *coarse) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t c = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         c < n_coarse; c += stride) {
        const int k0 = begin[c], k1 = begin[c + 1];
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int k = k0; k < k1; ++k) {
            const float4 v = *reinterpret_cast<const float4 *>(fine + 4 * static_cast<std::int64_t>(__ldg(children + k)));
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
        }
        *reinterpret_cast<float4 *>(coarse + 4 * c) = acc;
    }
}

template <typename T, bool ADD>
__global__ void prolong_kernel(const int *coarse_of, const T *w, std::int64_t n_fine,
                               const T *coarse, std::int64_t ldc, T *fine, std::int64_t ldf,
                               int nb) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         i < n_fine; i += stride) {
        const int c = coarse_of[i];
        const T wi = w[i];
        for (int col = 0; col < nb; ++col) {
            const T e = c >= 0 ? wi * coarse[c + col * ldc] : T(0);
            if constexpr (ADD) {
                fine[i + col * ldf] += e;
            } else {
                fine[i + col * ldf] = e;
            }
        }
    }
}

template <bool ADD>
__global__ void prolong_lanes_kernel(const int *coarse_of, const float *w, std::int64_t n_fine,
                                     const float *coarse, float *fine) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         i < n_fine; i += stride) {
        const int c = coarse_of[i];
        const float wi = w[i];
        float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c >= 0) {
            const float4 v = *reinterpret_cast<const float4 *>(coarse + 4 * static_cast<std::int64_t>(c));
            e = make_float4(wi * v.x, wi * v.y, wi * v.z, wi * v.w);
        }
        float4 *f = reinterpret_cast<float4 *>(fine + 4 * i);
        if constexpr (ADD) {
            const float4 o = *f;
            e = make_float4(o.x + e.x, o.y + e.y, o.z + e.z, o.w + e.w);
        }
        *f = e;
    }
}

std::size_t cub_bytes(std::int64_t n) {
    std::size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const int *>(nullptr),
                                    static_cast<int *>(nullptr), static_cast<const int *>(nullptr),
                                    static_cast<int *>(nullptr), static_cast<int>(n));
    return bytes;
}

std::size_t align256(std::size_t b) { return (b + 255) / 256 * 256; }

} // namespace

std::size_t children_scratch_bytes(std::int64_t n_fine) {
    // sorted keys, the iota values, CUB's own temporary storage
    return 2 * align256(static_cast<std::size_t>(n_fine) * sizeof(int)) + align256(cub_bytes(n_fine));
}

cudaError_t build_children(const int *coarse_of, std::int64_t n_fine, std::int64_t n_coarse,
                           int *children, int *begin, void *scratch, std::size_t scratch_bytes,
                           cudaStream_t stream) {
    if (n_fine <= 0 || n_fine >= (std::int64_t(1) << 31) || n_coarse < 0 ||
        scratch_bytes < children_scratch_bytes(n_fine)) {
        return cudaErrorInvalidValue;
    }
    auto *base = static_cast<unsigned char *>(scratch);
    int *keys = reinterpret_cast<int *>(base);
    int *ids = reinterpret_cast<int *>(base + align256(static_cast<std::size_t>(n_fine) * sizeof(int)));
    void *temp = base + 2 * align256(static_cast<std::size_t>(n_fine) * sizeof(int));
    std::size_t temp_bytes = cub_bytes(n_fine);
    count_launches(1);
    iota_kernel<<<grid_for(n_fine), kThreads, 0, stream>>>(ids, n_fine);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return e;
    }
    // a stable radix sort: equal keys keep ascending fine indices
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, coarse_of, keys, ids, children,
                                        static_cast<int>(n_fine), 0, static_cast<int>(sizeof(int) * 8),
                                        stream);
    if (e != cudaSuccess) {
        return e;
    }
    count_launches(1);
    bounds_kernel<<<grid_for(n_coarse + 1), kThreads, 0, stream>>>(keys, n_fine, n_coarse, begin);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_restrict(const int *begin, const int *children, std::int64_t n_coarse,
                            const T *fine, std::int64_t ld_fine, T *coarse, std::int64_t ld_coarse,
                            int nb, bool interleaved, cudaStream_t stream) {
    if (n_coarse == 0) {
        return cudaSuccess;
    }
    count_launches(1);
    if constexpr (std::is_same_v<T, float>) {
        if (interleaved) {
            restrict_lanes_kernel<<<grid_for(n_coarse), kThreads, 0, stream>>>(begin, children, n_coarse,
                                                                                fine, coarse);
            return cudaGetLastError();
        }
    }
    restrict_kernel<T><<<grid_for(n_coarse), kThreads, 0, stream>>>(begin, children, n_coarse, fine,
                                                                    ld_fine, coarse, ld_coarse, nb);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_prolong(const int *coarse_of, const T *weight, std::int64_t n_fine,
                           const T *coarse, std::int64_t ld_coarse, T *fine, std::int64_t ld_fine,
                           int nb, bool interleaved, bool add, cudaStream_t stream) {
    if (n_fine == 0) {
        return cudaSuccess;
    }
    count_launches(1);
    if constexpr (std::is_same_v<T, float>) {
        if (interleaved) {
            if (add) {
                prolong_lanes_kernel<true><<<grid_for(n_fine), kThreads, 0, stream>>>(coarse_of, weight, n_fine,
                                                                                       coarse, fine);
            } else {
                prolong_lanes_kernel<false><<<grid_for(n_fine), kThreads, 0, stream>>>(coarse_of, weight, n_fine,
                                                                                        coarse, fine);
            }
            return cudaGetLastError();
        }
    }
    if (add) {
        prolong_kernel<T, true><<<grid_for(n_fine), kThreads, 0, stream>>>(coarse_of, weight, n_fine, coarse,
                                                                           ld_coarse, fine, ld_fine, nb);
    } else {
        prolong_kernel<T, false><<<grid_for(n_fine), kThreads, 0, stream>>>(coarse_of, weight, n_fine, coarse,
                                                                            ld_coarse, fine, ld_fine, nb);
    }
    return cudaGetLastError();
}

template cudaError_t launch_restrict<double>(const int *, const int *, std::int64_t, const double *,
                                             std::int64_t, double *, std::int64_t, int, bool, cudaStream_t);
template cudaError_t launch_restrict<float>(const int *, const int *, std::int64_t, const float *,
                                            std::int64_t, float *, std::int64_t, int, bool, cudaStream_t);
template cudaError_t launch_prolong<double>(const int *, const double *, std::int64_t, const double *,
                                            std::int64_t, double *, std::int64_t, int, bool, bool, cudaStream_t);
template cudaError_t launch_prolong<float>(const int *, const float *, std::int64_t, const float *,
                                           std::int64_t, float *, std::int64_t, int, bool, bool, cudaStream_t);

} // namespace mkb
