// The assembled generator (markovkit/generator.hpp:84-107): generator::matrix() = Q and
// characteristic_matrix(shift) = shift I - Q as CSR in device memory, and n_jumps() (:48).
#pragma once

#include "engine.hpp"

namespace mkb {

// sign * (Q - shift I) with 64-bit indices: each row's columns ascending, and the rates of
// distinct jumps between one pair of states summed into one entry, as the reference's
// num::spmat::from_triplets does with its triplets.
struct Csr {
    std::int64_t rows = 0;
    std::int64_t nnz = 0;
    DeviceArray<std::int64_t> row_ptr; // rows + 1
    DeviceArray<std::int64_t> col;     // nnz
    DeviceArray<double> val;           // nnz
};

// matrix(): shift 0, sign 1; characteristic_matrix(s): shift s, sign -1 (generator.hpp:93-107)
void assemble(const Generator &g, double shift, double sign, Csr &out, cudaStream_t stream);

// n_jumps(): the jumps that stay in the space, one per (source state, transition)
std::int64_t count_jumps(const Generator &g, cudaStream_t stream);

} // namespace mkb
