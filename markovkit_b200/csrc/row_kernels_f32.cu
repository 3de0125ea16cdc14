// FP32 instantiations of the row kernels (row_kernels_impl.cuh), one right-hand side.
#include "row_kernels_impl.cuh"

namespace mkb {

cudaError_t launch_rows_f32(const RowParams<float> &p, int S, int cap, cudaStream_t stream) {
    if (p.nb > 1) {
        return launch_rows_f32_batch(p, S, cap, stream);
    }
    return launch_rows_impl<float, 1>(p, S, cap, stream);
}

} // namespace mkb
