// Arithmetic numbering of RDME population states, shared by host set-up code and sm_100a
// kernels.
//
// MarkovKit numbers the states of one population sector lexicographically: species 0 is
// the most significant digit, and inside one species the count in voxel 0 is the most
// significant, ascending (markovkit/rdme/population_space.hpp:32-72, rank at :75-100).
// The reference walks all V voxels per species to rank a state. Here a species'
// composition is held as its molecules instead: u = V - 1 - voxel for each molecule,
// sorted ascending. A composition is a stars-and-bars string whose lexicographic order is
// exactly the order above, and the rank of such a string is the combinatorial number
//     rank = sum_{p=0}^{t-1} C(u_p + p, p + 1),
// so ranking costs O(t) instead of O(V), and unranking is t searches in binomial rows.
// Both are bit-exact with population_space.hpp's rank / enumerate (checked in the tests
// against every state of the reference's own enumeration).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define MK_HD __host__ __device__ __forceinline__
#else
#define MK_HD inline
#endif

namespace mkb {

constexpr int kMaxSpecies = 4;
constexpr int kMaxReactions = 16;

// C(q, j) for 0 <= j <= jmax, 0 <= q <= qmax, row-major by j; entries saturate at 2^62
struct BinomTable {
    const std::int64_t *data = nullptr;
    int jmax = 0;
    int qmax = 0;
};

MK_HD std::int64_t binom(const BinomTable &B, int q, int j) {
    if (q < 0 || j < 0 || q > B.qmax || j > B.jmax) {
        return 0;
    }
#if defined(__CUDA_ARCH__)
    return __ldg(B.data + static_cast<std::int64_t>(j) * (B.qmax + 1) + q);
#else
    return B.data[static_cast<std::int64_t>(j) * (B.qmax + 1) + q];
#endif
}

// u[0..t) (ascending) of the composition with rank r among compositions of t into V voxels
MK_HD void unrank_species(const BinomTable &B, std::int64_t r, int t, int V, int *u) {
    int hi = (V - 1) + (t - 1);
    for (int j = t; j >= 1; --j) {
        int lo = j - 1;
        int h = hi;
        while (lo < h) {
            const int mid = (lo + h + 1) >> 1;
            if (binom(B, mid, j) <= r) {
                lo = mid;
            } else {
                h = mid - 1;
            }
        }
        u[j - 1] = lo - (j - 1);
        r -= binom(B, lo, j);
        hi = lo - 1;
    }
}

// rank of an ascending molecule list
MK_HD std::int64_t rank_species(const BinomTable &B, const int *u, int t) {
    std::int64_t r = 0;
    for (int p = 0; p < t; ++p) {
        r += binom(B, u[p] + p, p + 1);
    }
    return r;
}

// rank of the list with one copy of u_rm removed and one copy of u_add inserted
MK_HD std::int64_t rank_replace(const BinomTable &B, const int *u, int t, int u_rm, int u_add) {
    std::int64_t r = 0;
    int p = 0;
    bool removed = false, added = false;
    for (int i = 0; i < t; ++i) {
        const int val = u[i];
        if (!added && u_add <= val) {
            r += binom(B, u_add + p, p + 1);
            ++p;
            added = true;
        }
        if (!removed && val == u_rm) {
            removed = true;
            continue;
        }
        r += binom(B, val + p, p + 1);
        ++p;
    }
    if (!added) {
        r += binom(B, u_add + p, p + 1);
    }
    return r;
}

// rank of the list with the multiplicity of value u changed by delta (delta < 0 removes)
MK_HD std::int64_t rank_modified(const BinomTable &B, const int *u, int t, int value, int delta) {
    std::int64_t r = 0;
    int p = 0;
    int skip = delta < 0 ? -delta : 0;
    int add = delta > 0 ? delta : 0;
    for (int i = 0; i < t; ++i) {
        const int val = u[i];
        while (add > 0 && value <= val) {
            r += binom(B, value + p, p + 1);
            ++p;
            --add;
        }
        if (skip > 0 && val == value) {
            --skip;
            continue;
        }
        r += binom(B, val + p, p + 1);
        ++p;
    }
    while (add > 0) {
        r += binom(B, value + p, p + 1);
        ++p;
        --add;
    }
    return r;
}

// how many entries of the ascending list equal value
MK_HD int count_of(const int *u, int t, int value) {
    int c = 0;
    for (int i = 0; i < t; ++i) {
        c += (u[i] == value) ? 1 : 0;
    }
    return c;
}

// One population sector inside a level space: all states with these species totals,
// numbered from `begin` in the reference's order.
struct SectorDesc {
    std::int64_t begin = 0;
    std::int64_t size = 0;
    std::int64_t stride[kMaxSpecies] = {}; // mixed-radix weight of species s's rank
    int total[kMaxSpecies] = {};
    int mol_offset[kMaxSpecies] = {}; // where species s starts in the molecule list
    int n_mol = 0;                    // molecules in a state of this sector
    int src[kMaxReactions] = {};      // sector holding the source of an in-jump of reaction r
    int dst[kMaxReactions] = {};      // sector reached by reaction r, -1 outside the space
    int heavy = 0;                    // some in-jump reaction can start at an empty voxel
    int coarse = -1;                  // slot of the same totals on the next multigrid level
    int terminal = -1;                // dense terminal block of this sector, -1 if none
    int pad = 0;
};

// decompose a local index into species ranks (species 0 most significant)
MK_HD void split_local(const SectorDesc &sec, int S, std::int64_t local, std::int64_t *rank) {
    std::int64_t rem = local;
    for (int s = 0; s < S; ++s) {
        if (s + 1 == S) {
            rank[s] = rem;
        } else {
            rank[s] = rem / sec.stride[s];
            rem -= rank[s] * sec.stride[s];
        }
    }
}

} // namespace mkb
