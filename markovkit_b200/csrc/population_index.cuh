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
// so ranking costs O(t) instead of O(V), and unranking is t inversions of C(., j).
// Both are bit-exact with population_space.hpp's rank / enumerate (checked in the tests
// against every state of the reference's own enumeration).
//
// Loops over molecules run to a compile-time bound TMAX with a runtime guard, so that after
// unrolling every array index is static and the molecule lists stay in registers.
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>

#if defined(__CUDACC__)
#define MK_HD __host__ __device__ __forceinline__
#else
#define MK_HD inline
#endif

#if defined(__CUDACC__) || defined(__clang__)
#define MK_PRAGMA(x) _Pragma(#x)
#else
#define MK_PRAGMA(x)
#endif
// unroll small molecule loops fully; leave long ones as loops
#define MK_UNROLL_MOL MK_PRAGMA(unroll(TMAX <= 8 ? TMAX : 1))

namespace mkb {

constexpr int kMaxSpecies = 4;
constexpr int kMaxReactions = 16;

// C(q, j) for 0 <= j <= jmax, 0 <= q <= qmax, row-major by j; entries saturate at 2^62
struct BinomTable {
    const std::int64_t *data = nullptr;
    int jmax = 0;
    int qmax = 0;
};

MK_HD std::int64_t binom_table(const BinomTable &B, int q, int j) {
    if (q < 0 || j < 0 || q > B.qmax || j > B.jmax) {
        return 0;
    }
#if defined(__CUDA_ARCH__)
    return __ldg(B.data + static_cast<std::int64_t>(j) * (B.qmax + 1) + q);
#else
    return B.data[static_cast<std::int64_t>(j) * (B.qmax + 1) + q];
#endif
}

// f(std::integral_constant<int, i>) for i = 0 .. N-1, unrolled at compile time
template <int N, typename F>
MK_HD void static_for(F &&f) {
    if constexpr (N > 0) {
        static_for<N - 1>(f);
        f(std::integral_constant<int, N - 1>{});
    }
}

// C(q, J) for a compile-time order J <= 4 (q >= 0, q < 2^14 when J > 2)
template <int J>
MK_HD std::int64_t binom_j(int q) {
    const std::int64_t Q = q;
    if constexpr (J == 0) {
        return 1;
    } else if constexpr (J == 1) {
        return Q;
    } else if constexpr (J == 2) {
        return (Q * (Q - 1)) >> 1;
    } else if constexpr (J == 3) {
        return (Q * (Q - 1) * (Q - 2)) / 6;
    } else {
        return (Q * (Q - 1) * (Q - 2) * (Q - 3)) / 24;
    }
}

// C(q, j): exact arithmetic for j <= 4 and q < 2^14 (the common case), else the table
MK_HD std::int64_t binom(const BinomTable &B, int q, int j) {
    if (q < j || j < 0) {
        return 0;
    }
    if (j <= 2) {
        return j == 0 ? 1 : (j == 1 ? std::int64_t(q) : (std::int64_t(q) * (q - 1)) >> 1);
    }
    if (q < 16384) {
        const std::int64_t Q = q;
        switch (j) {
        case 0:
            return 1;
        case 1:
            return Q;
        case 2:
            return (Q * (Q - 1)) >> 1;
        case 3:
            return (Q * (Q - 1) * (Q - 2)) / 6;
        case 4:
            return (Q * (Q - 1) * (Q - 2) * (Q - 3)) / 24;
        default:
            break;
        }
    }
    return binom_table(B, q, j);
}

// largest q in [j - 1, hi] with C(q, j) <= r, from a floating-point estimate
MK_HD int inverse_binom(const BinomTable &B, std::int64_t r, int j, int hi) {
    if (j == 1) {
        return static_cast<int>(r < hi ? r : hi);
    }
    double est;
    if (j == 2) {
        est = std::floor(0.5 * (1.0 + std::sqrt(1.0 + 8.0 * static_cast<double>(r))));
    } else {
        double fact = 1.0;
        for (int k = 2; k <= j; ++k) {
            fact *= k;
        }
        est = std::pow(fact * static_cast<double>(r), 1.0 / j) + 0.5 * (j - 1);
    }
    int q = est < static_cast<double>(j - 1) ? j - 1 : (est > static_cast<double>(hi) ? hi : static_cast<int>(est));
    while (q < hi && binom(B, q + 1, j) <= r) {
        ++q;
    }
    while (q > j - 1 && binom(B, q, j) > r) {
        --q;
    }
    return q;
}

// u[0..t) (ascending) of the composition with rank r among compositions of t into V voxels
template <int TMAX>
MK_HD void unrank_species(const BinomTable &B, std::int64_t r, int t, int V, int (&u)[TMAX]) {
    int hi = (V - 1) + (t - 1);
    MK_UNROLL_MOL
    for (int k = TMAX; k >= 1; --k) {
        if (k <= t) {
            const int q = inverse_binom(B, r, k, hi);
            u[k - 1] = q - (k - 1);
            r -= binom(B, q, k);
            hi = q - 1;
        }
    }
}

// rank of an ascending molecule list
template <int TMAX>
MK_HD std::int64_t rank_species(const BinomTable &B, const int (&u)[TMAX], int t) {
    std::int64_t r = 0;
    MK_UNROLL_MOL
    for (int p = 0; p < TMAX; ++p) {
        if (p < t) {
            r += binom(B, u[p] + p, p + 1);
        }
    }
    return r;
}

// C(u + p, p + 1) for a position p known to lie in [P - 1, P + 1], P compile-time: the three
// candidates have compile-time orders, so no branch on p is needed
template <int P>
MK_HD std::int64_t binom_at(int u, int p) {
    const std::int64_t mid = binom_j<(P + 1 <= 4 ? P + 1 : 4)>(u + P);
    std::int64_t lo = 0, hi = 0;
    if constexpr (P >= 1) {
        lo = binom_j<P>(u + P - 1);
    }
    if constexpr (P + 2 <= 4) {
        hi = binom_j<P + 2>(u + P + 1);
    }
    return p == P ? mid : (p < P ? lo : hi);
}

// rank of the list with one copy of u_rm removed and one copy of u_add inserted
template <int TMAX>
MK_HD std::int64_t rank_replace(const BinomTable &B, const int (&u)[TMAX], int t, int u_rm,
                                int u_add) {
    if constexpr (TMAX == 1) {
        // the only molecule moves: the new list is {u_add}
        return u_add;
    } else if constexpr (TMAX == 2) {
        // at most two molecules: the one that stays, o, and u_add, ranked in closed form
        if (t < 2) {
            return u_add;
        }
        const int o = u[0] == u_rm ? u[1] : u[0];
        const int a = o < u_add ? o : u_add, b = o < u_add ? u_add : o;
        return a + ((std::int64_t(b) * (b + 1)) >> 1);
    } else if constexpr (TMAX <= 4) {
        // branch-free for short lists: element i (not the removed copy a) lands at
        // i - [i > a] + [u_i >= u_add]; u_add lands after the b remaining smaller elements
        int a = -1;
#pragma unroll
        for (int i = 0; i < TMAX; ++i) {
            a = (i < t && u[i] == u_rm) ? i : a;
        }
        int b = 0;
#pragma unroll
        for (int i = 0; i < TMAX; ++i) {
            b += (i < t && i != a && u[i] < u_add) ? 1 : 0;
        }
        std::int64_t r = 0;
        static_for<TMAX>([&](auto I) {
            constexpr int i = decltype(I)::value;
            if (i < t && i != a) {
                const int pos = i - (i > a ? 1 : 0) + (u[i] >= u_add ? 1 : 0);
                r += binom_at<i>(u[i], pos);
            }
        });
        std::int64_t add = 0;
        static_for<TMAX>([&](auto Q) {
            constexpr int q = decltype(Q)::value;
            add = (b == q) ? binom_j<(q + 1 <= 4 ? q + 1 : 4)>(u_add + q) : add;
        });
        return r + add;
    }
    std::int64_t r = 0;
    int p = 0;
    bool removed = false, added = false;
    MK_UNROLL_MOL
    for (int i = 0; i < TMAX; ++i) {
        if (i < t) {
            const int val = u[i];
            if (!added && u_add <= val) {
                r += binom(B, u_add + p, p + 1);
                ++p;
                added = true;
            }
            if (!removed && val == u_rm) {
                removed = true;
            } else {
                r += binom(B, val + p, p + 1);
                ++p;
            }
        }
    }
    if (!added) {
        r += binom(B, u_add + p, p + 1);
    }
    return r;
}

// rank of the list with the multiplicity of `value` changed by delta (delta < 0 removes)
template <int TMAX>
MK_HD std::int64_t rank_modified(const BinomTable &B, const int (&u)[TMAX], int t, int value,
                                 int delta) {
    if constexpr (TMAX <= 2) {
        // lists of at most two molecules before and after: closed forms for one copy more/less
        if (delta == 1) {
            if (t == 0) {
                return value;
            }
            const int a = u[0] < value ? u[0] : value, b = u[0] < value ? value : u[0];
            return a + ((std::int64_t(b) * (b + 1)) >> 1);
        }
        if (delta == -1) {
            return t == 2 ? (u[0] == value ? u[TMAX - 1] : u[0]) : 0;
        }
    }
    std::int64_t r = 0;
    int p = 0;
    int skip = delta < 0 ? -delta : 0;
    int add = delta > 0 ? delta : 0;
    MK_UNROLL_MOL
    for (int i = 0; i < TMAX; ++i) {
        if (i < t) {
            const int val = u[i];
            while (add > 0 && value <= val) {
                r += binom(B, value + p, p + 1);
                ++p;
                --add;
            }
            if (skip > 0 && val == value) {
                --skip;
            } else {
                r += binom(B, val + p, p + 1);
                ++p;
            }
        }
    }
    while (add > 0) {
        r += binom(B, value + p, p + 1);
        ++p;
        --add;
    }
    return r;
}

// how many entries of the list equal value
template <int TMAX>
MK_HD int count_of(const int (&u)[TMAX], int t, int value) {
    int c = 0;
    MK_UNROLL_MOL
    for (int i = 0; i < TMAX; ++i) {
        c += (i < t && u[i] == value) ? 1 : 0;
    }
    return c;
}

// One population sector inside a level space: all states with these species totals,
// numbered from `begin` in the reference's order.
struct SectorDesc {
    std::int64_t begin = 0;
    std::int64_t size = 0;
    std::int64_t stride[kMaxSpecies] = {}; // mixed-radix weight of species s's rank
    double inv_stride[kMaxSpecies] = {};   // 1 / stride, for division by multiplication
    int total[kMaxSpecies] = {};
    int mol_offset[kMaxSpecies] = {}; // where species s starts in a flat molecule list
    int n_mol = 0;                    // molecules in a state of this sector
    int src[kMaxReactions] = {};      // sector holding the source of an in-jump of reaction r
    int dst[kMaxReactions] = {};      // sector reached by reaction r, -1 outside the space
    int heavy = 0;                    // some in-jump reaction can start at an empty voxel
    int coarse = -1;                  // slot of the same totals on the next multigrid level
    int terminal = -1;                // dense terminal block of this sector, -1 if none
    int gs_class = 0;                 // full-operator Gauss-Seidel: the sector's colour class
};

// q = floor(a / b) for 0 <= a < 2^52, b >= 1, from a * (1/b) in double and one correction
// (the product is within one unit of a / b)
MK_HD std::int64_t div_floor(std::int64_t a, std::int64_t b, double inv_b) {
    std::int64_t q = static_cast<std::int64_t>(static_cast<double>(a) * inv_b);
    if (q * b > a) {
        --q;
    } else if ((q + 1) * b <= a) {
        ++q;
    }
    return q;
}

// decompose a local index into species ranks (species 0 most significant)
MK_HD void split_local(const SectorDesc &sec, int S, std::int64_t local, std::int64_t (&rank)[kMaxSpecies]) {
    std::int64_t rem = local;
#pragma unroll
    for (int s = 0; s < kMaxSpecies; ++s) {
        if (s < S) {
            if (s + 1 == S) {
                rank[s] = rem;
            } else {
                rank[s] = div_floor(rem, sec.stride[s], sec.inv_stride[s]);
                rem -= rank[s] * sec.stride[s];
            }
        } else {
            rank[s] = 0;
        }
    }
}

} // namespace mkb
