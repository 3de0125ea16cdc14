// FP64 instantiations of the row kernels (row_kernels_impl.cuh), one right-hand side.
#include "row_kernels_impl.cuh"

namespace mkb {

cudaError_t launch_rows_f64(const RowParams<double> &p, int S, int cap, cudaStream_t stream) {
    if (p.nb > 1) {
        return launch_rows_f64_batch(p, S, cap, stream);
    }
    return launch_rows_impl<double, 1>(p, S, cap, stream);
}

} // namespace mkb
