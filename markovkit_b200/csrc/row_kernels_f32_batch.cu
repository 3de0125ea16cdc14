// FP32 instantiations of the row kernels (row_kernels_impl.cuh) for up to kRowBatch
// right-hand sides at once.
#include "row_kernels_impl.cuh"

namespace mkb {

cudaError_t launch_rows_f32_batch(const RowParams<float> &p, int S, int cap, cudaStream_t stream) {
    if (p.nb < 1 || p.nb > kRowBatch) {
        return cudaErrorInvalidValue;
    }
    return launch_rows_impl<float, kRowBatch>(p, S, cap, stream);
}

} // namespace mkb
