// FP32 instantiations of the row kernels (row_kernels_impl.cuh), for the FP32 multigrid.
#include "row_kernels_impl.cuh"

namespace mkb {

cudaError_t launch_rows_f32(const RowParams<float> &p, int S, int cap, cudaStream_t stream) {
    return launch_rows_impl<float>(p, S, cap, stream);
}

} // namespace mkb
