// Dense inverses of a multigrid level's terminal blocks (the sectors a level solves directly,
// markovkit/rdme/multigrid.hpp:309-317 factors them densely): Gauss-Jordan elimination with
// partial pivoting on [A | I], the same steps and the same roundings as the host routine it
// replaces (each update a separate multiply and subtract, IEEE division), so the inverse is
// bit-identical; it runs on the device when the blocks are large enough for the O(n^3) work
// to matter (a 13-voxel terminal grid with lists of four molecules has blocks of 1820 states).
#pragma once

#include <cstdint>
#include <vector>

namespace mkb {

// Blocks b = 0.. of sizes n[b], stored row-major in A at offset[b] (n[b]^2 entries each);
// inv receives the inverses at the same offsets. Returns false when a block is singular (a
// zero pivot). A is left in an unspecified state.
bool invert_dense_blocks(std::vector<double> &A, const std::vector<std::int64_t> &offset,
                         const std::vector<int> &n, std::vector<double> &inv);

// the host routine on one block (A overwritten); false when singular
bool invert_dense(std::vector<double> &A, int n, std::vector<double> &inv);

} // namespace mkb
