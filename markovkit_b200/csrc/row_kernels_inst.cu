// One explicit instantiation of the general row kernel (row_kernels_impl.cuh): the build
// compiles this file once per (precision MK_T, batch width MK_NB, state shape MK_SHAPE), so the
// instantiations compile in parallel. MK_SHAPE indexes the shapes of with_shape
// (generator_row.cuh).
#include "row_kernels_impl.cuh"

#if !defined(MK_T) || !defined(MK_NB) || !defined(MK_SHAPE)
#error "compile with -DMK_T=<double|float> -DMK_NB=<1|4> -DMK_SHAPE=<0..9>"
#endif

namespace mkb::detail {

#if MK_SHAPE == 0
template cudaError_t launch_shape<MK_T, 1, 2, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 1
template cudaError_t launch_shape<MK_T, 1, 4, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 2
template cudaError_t launch_shape<MK_T, 1, 16, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 3
template cudaError_t launch_shape<MK_T, 1, 64, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 4
template cudaError_t launch_shape<MK_T, 2, 1, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 5
template cudaError_t launch_shape<MK_T, 2, 2, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 6
template cudaError_t launch_shape<MK_T, 2, 4, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 7
template cudaError_t launch_shape<MK_T, 2, 16, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 8
template cudaError_t launch_shape<MK_T, kMaxSpecies, 4, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#elif MK_SHAPE == 9
template cudaError_t launch_shape<MK_T, kMaxSpecies, 16, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
#else
#error "MK_SHAPE out of range"
#endif

} // namespace mkb::detail
