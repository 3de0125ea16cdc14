// Multigrid transfers between a level and the next coarser one, in a fixed order so that every
// cycle is bitwise reproducible whatever else runs on the device
// (population_transfer::restrict / prolong, markovkit/rdme/multigrid.hpp:100-111):
//  * restriction: coarse_c = sum of the fine children of c, added in ascending fine index;
//  * prolongation: fine_i (+)= w_i coarse_{c(i)}, a gather with the weights stored at set-up.
// The children lists come from one stable sort of the fine states by coarse state.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mkb {

// scratch bytes build_children needs for n_fine fine states
std::size_t children_scratch_bytes(std::int64_t n_fine);

// children[begin[c] .. begin[c + 1]) = the fine states whose coarse_of is c, ascending, for
// c < n_coarse (fine states with coarse_of < 0 sit before begin[0]); scratch of
// children_scratch_bytes(n_fine) bytes
cudaError_t build_children(const int *coarse_of, std::int64_t n_fine, std::int64_t n_coarse,
                           int *children, int *begin, void *scratch, std::size_t scratch_bytes,
                           cudaStream_t stream);

// coarse = R fine for nb columns (column c at c * ld; interleaved: the FP32 batch's four
// lanes of entry i at 4 i .. 4 i + 3, all lanes summed)
template <typename T>
cudaError_t launch_restrict(const int *begin, const int *children, std::int64_t n_coarse,
                            const T *fine, std::int64_t ld_fine, T *coarse, std::int64_t ld_coarse,
                            int nb, bool interleaved, cudaStream_t stream);

// fine = P coarse (add: fine += P coarse); fine states without a coarse state get 0 (add: keep)
template <typename T>
cudaError_t launch_prolong(const int *coarse_of, const T *weight, std::int64_t n_fine,
                           const T *coarse, std::int64_t ld_coarse, T *fine, std::int64_t ld_fine,
                           int nb, bool interleaved, bool add, cudaStream_t stream);

} // namespace mkb
