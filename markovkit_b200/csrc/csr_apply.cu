// A caller-given sparse matrix in CSR on the device and y = shift x + sign A x over it: the
// generator of an FSP support or any other explicitly listed chain (generator.hpp:27-44 builds
// such a Q from a state list), applied by the C ABI's mk_csr_apply.
#include "capi_internal.hpp"
#include "launch_count.hpp"

#include <algorithm>
#include <vector>

using namespace mkb;
using mkb::capi::as_stream;
using mkb::capi::guarded;

namespace {

constexpr int kCsrThreads = 256;

// a warp per row: lanes stride the row's entries, partial sums meet by shuffles
__global__ void __launch_bounds__(kCsrThreads)
    csr_apply_kernel(const std::int64_t *__restrict__ ptr, const std::int64_t *__restrict__ col,
                     const double *__restrict__ val, std::int64_t rows, double shift, double sign,
                     const double *__restrict__ x, double *__restrict__ y) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const std::int64_t warps = static_cast<std::int64_t>(gridDim.x) * (kCsrThreads / 32);
    for (std::int64_t r = (blockIdx.x * static_cast<std::int64_t>(kCsrThreads) + threadIdx.x) / 32;
         r < rows; r += warps) {
        double s = 0.0;
        for (std::int64_t p = ptr[r] + lane; p < ptr[r + 1]; p += 32) {
            s = fma(val[p], x[col[p]], s);
        }
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffU, s, o);
        }
        if (lane == 0) {
            y[r] = shift * x[r] + sign * s;
        }
    }
}

} // namespace

int mk_csr_create_host(int64_t rows, const int64_t *row_ptr, const int64_t *col, const double *val,
                       mk_csr *out) {
    return guarded([&] {
        MK_REQUIRE(row_ptr && out && rows >= 0, "null argument");
        MK_REQUIRE(row_ptr[0] == 0, "csr: row_ptr[0] must be 0");
        for (int64_t r = 0; r < rows; ++r) {
            MK_REQUIRE(row_ptr[r + 1] >= row_ptr[r], "csr: row pointers must not decrease");
        }
        const int64_t nnz = row_ptr[rows];
        MK_REQUIRE(nnz == 0 || (col && val), "null argument");
        for (int64_t p = 0; p < nnz; ++p) {
            MK_REQUIRE(col[p] >= 0 && col[p] < rows, "csr: column out of range");
        }
        auto h = std::make_unique<mk_csr_s>();
        h->csr.rows = rows;
        h->csr.nnz = nnz;
        h->csr.row_ptr.upload(std::vector<std::int64_t>(row_ptr, row_ptr + rows + 1));
        h->csr.col.upload(std::vector<std::int64_t>(col, col + nnz));
        h->csr.val.upload(std::vector<double>(val, val + nnz));
        *out = h.release();
    });
}

int mk_csr_apply(mk_csr m, double shift, double sign, const double *d_x, double *d_y, void *stream) {
    return guarded([&] {
        MK_REQUIRE(m && d_x && d_y, "null argument");
        const auto &c = m->csr;
        if (c.rows == 0) {
            return;
        }
        const std::int64_t blocks = std::clamp<std::int64_t>((c.rows * 32 + kCsrThreads - 1) / kCsrThreads, 1,
                                                             148 * 16);
        count_launches(1);
        csr_apply_kernel<<<static_cast<unsigned>(blocks), kCsrThreads, 0, as_stream(stream)>>>(
            c.row_ptr.get(), c.col.get(), c.val.get(), c.rows, shift, sign, d_x, d_y);
        check_cuda(cudaGetLastError(), "csr apply");
    });
}
