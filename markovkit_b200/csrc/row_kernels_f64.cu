// FP64 instantiations of the row kernels (row_kernels_impl.cuh).
#include "row_kernels_impl.cuh"

namespace mkb {

cudaError_t launch_rows_f64(const RowParams<double> &p, int S, int cap, cudaStream_t stream) {
    return launch_rows_impl<double>(p, S, cap, stream);
}

} // namespace mkb
