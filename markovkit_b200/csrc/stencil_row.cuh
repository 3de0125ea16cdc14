// Rows of structured-grid levels for the state shapes of the solve workloads: one species of at
// most four molecules, or two species of at most one each. The terms, their values and their
// order are those of visit_row (generator_row.cuh) for a light row, so the results are
// bit-identical; what changes is how the row gets there:
//  * the state is unranked with closed-form estimates of the combinatorial number system
//    (single-precision root, then an exact integer correction) instead of the table search;
//  * each molecule's voxel is read once from a per-voxel mask (which neighbours exist along each
//    axis, and the voxel's checkerboard colour) instead of coordinates and boundary tests;
//  * an in-jump's source rank is a closed form of the molecule that moves: row +- stride for a
//    lone molecule, min + max(max + 1) / 2 for a pair, a binomial difference for longer lists.
// Rows whose in-jumps fan in from every voxel ("heavy" rows) keep the general kernel.
#pragma once

#include "generator_row.cuh"

#include <math.h>

namespace mkb {

// largest q in [J - 1, hi] with C(q, J) <= r for J <= 4 and r < 2^31 (ranks inside a level
// space): a single-precision estimate of the root, corrected in exact integer arithmetic
template <int J>
MK_HD int inverse_binom_small(std::int64_t r, int hi) {
    static_assert(J >= 1 && J <= 4, "orders 1..4");
    if constexpr (J == 1) {
        return static_cast<int>(r < hi ? r : hi);
    } else {
        const float fr = static_cast<float>(r);
        float est;
        if constexpr (J == 2) {
            est = 0.5f * (1.0f + sqrtf(8.0f * fr + 1.0f)); // C(q, 2) = q (q - 1) / 2
        } else if constexpr (J == 3) {
            est = cbrtf(6.0f * fr) + 1.0f; // C(q, 3) ~ (q - 1)^3 / 6
        } else {
            est = sqrtf(sqrtf(24.0f * fr)) + 1.5f; // C(q, 4) ~ (q - 3/2)^4 / 24
        }
        int q = est < static_cast<float>(J - 1)
                    ? J - 1
                    : (est > static_cast<float>(hi) ? hi : static_cast<int>(est));
        while (q < hi && binom_j<J>(q + 1) <= r) {
            ++q;
        }
        while (q > J - 1 && binom_j<J>(q) > r) {
            --q;
        }
        return q;
    }
}

// u[0..t) (ascending) of the composition with rank r among compositions of t <= TMAX <= 4
// molecules into V voxels; the same list as unrank_species
template <int TMAX>
MK_HD void unrank_small(int r, int t, int V, int (&u)[TMAX]) {
    static_assert(TMAX >= 1 && TMAX <= 4, "short molecule lists only");
    std::int64_t rr = r;
    int hi = (V - 1) + (t - 1);
    static_for<TMAX>([&](auto I) {
        constexpr int k = TMAX - decltype(I)::value; // positions from the last one down
        u[k - 1] = 0;
        if (k <= t) {
            const int q = inverse_binom_small<k>(rr, hi);
            u[k - 1] = q - (k - 1);
            rr -= binom_j<k>(q);
            hi = q - 1;
        }
    });
}

// the unranked row and the mask of each molecule's voxel (0 for absent molecules)
template <int NS, int TMAX>
struct StencilState {
    RowState<NS, TMAX> rs;
    unsigned m[NS][TMAX];
};

template <typename T, int NS, int TMAX>
MK_HD void stencil_load(const SectorDesc &sec, const ModelView<T> &md, int local,
                        StencilState<NS, TMAX> &st) {
    split_species<NS>(sec, md.S, local, st.rs.rank);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int t = s < md.S ? sec.total[s] : 0;
        unrank_small<TMAX>(st.rs.rank[s], t, md.V, st.rs.u[s]);
#pragma unroll
        for (int p = 0; p < TMAX; ++p) {
            st.m[s][p] = p < t ? load_ro(md.vmask + (md.V - 1 - st.rs.u[s][p])) : 0U;
        }
    }
}

// checkerboard colour of the state (state_colour through the masks)
template <int NS, int TMAX>
MK_HD int stencil_colour(const StencilState<NS, TMAX> &st) {
    unsigned c = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
#pragma unroll
        for (int p = 0; p < TMAX; ++p) {
            c ^= st.m[s][p];
        }
    }
    return static_cast<int>((c >> kVoxelColourBit) & 1U);
}

// Diffusion of species s (diffusion_terms on a structured grid): each molecule's exit rate and
// the in-jumps into its voxel from the neighbours the mask lists, a run of equal molecules
// entered from above through its last copy and from below through its first.
template <typename T, int NS, int TMAX, bool WANT_IN, typename Acc>
MK_HD void stencil_diffusion(const SectorDesc &sec, const ModelView<T> &md,
                             const StencilState<NS, TMAX> &st, int s, int row, T &exit, Acc &acc) {
    const int t = sec.total[s];
    const T Ds = md.diff[s];
    const int stride = static_cast<int>(sec.stride[s]);
    const int(&u)[TMAX] = st.rs.u[s];
    const int rank = st.rs.rank[s];
    static_for<TMAX>([&](auto P) {
        constexpr int p = decltype(P)::value;
        if (p >= t) {
            return;
        }
        const int uu = u[p];
        const unsigned mk = st.m[s][p];
        const bool first = p == 0 || u[p > 0 ? p - 1 : 0] != uu;
        const bool last = p + 1 >= t || u[p + 1 < TMAX ? p + 1 : p] != uu;
        // the in-jump from the neighbour with reversed index uw (one copy of uu moved there)
        auto in_jump = [&](int uw, T coef) {
            int nw = 0;
            int delta;
            if constexpr (TMAX == 1) {
                delta = uw - uu;
            } else if constexpr (TMAX == 2) {
                if (t < 2) {
                    delta = uw - uu;
                } else {
                    const int o = p == 0 ? u[1] : u[0];
                    nw = o == uw ? 1 : 0;
                    const int a = o < uw ? o : uw, b = o < uw ? uw : o;
                    delta = static_cast<int>(a + ((std::int64_t(b) * (b + 1)) >> 1)) - rank;
                }
            } else {
                nw = count_of<TMAX>(u, t, uw);
                const int lo = p > 0 ? u[p > 0 ? p - 1 : 0] : -1;
                const int hi = p + 1 < t ? u[p + 1 < TMAX ? p + 1 : p] : 0x7fffffff;
                constexpr int J = p + 1 <= 4 ? p + 1 : 4;
                if (uw > uu ? uw <= hi : uw >= lo) {
                    delta = static_cast<int>(binom_j<J>(uw + p) - binom_j<J>(uu + p));
                } else {
                    delta = static_cast<int>(rank_replace<TMAX>(BinomTable{}, u, t, uu, uw)) - rank;
                }
            }
            const T rate = T(nw + 1) * Ds * coef;
            acc(row + delta * stride, rate, T(0));
        };
        T deg = T(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a >= md.grid_dim) {
                continue;
            }
            const bool has_lo = ((mk >> (2 * a)) & 1U) != 0;
            const bool has_hi = ((mk >> (2 * a + 1)) & 1U) != 0;
            deg += T((has_lo ? 1 : 0) + (has_hi ? 1 : 0)) * md.axis_coef[a];
            if constexpr (WANT_IN) {
                // neighbour v - stride has reversed index uu + stride, v + stride uu - stride
                if (has_lo && last) {
                    in_jump(uu + md.gstride[a], md.axis_coef[a]);
                }
                if (has_hi && first) {
                    in_jump(uu - md.gstride[a], md.axis_coef[a]);
                }
            }
        }
        exit += Ds * deg;
    });
}

// a light row (visit_row with light = true, one lane) through the stencil forms
template <typename T, int NS, int TMAX, bool WANT_IN, typename Acc>
MK_HD void stencil_visit(const BinomTable &B, const SectorDesc *sectors, const SectorDesc &sec,
                         const ModelView<T> &md, const StencilState<NS, TMAX> &st, int row,
                         T &exit, T &leak, Acc &&acc) {
    empty_reaction_terms<T>(sec, md, exit, leak);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (s < md.S && sec.total[s] > 0) {
            stencil_diffusion<T, NS, TMAX, WANT_IN>(sec, md, st, s, row, exit, acc);
        }
    }
    occupied_reaction_terms<T, NS, TMAX, WANT_IN>(B, sectors, sec, md, st.rs, exit, leak, acc);
}

// the shapes the stencil rows serve: (species S, largest species total cap) -> (NS, TMAX);
// f.template operator()<NS, TMAX>() as with_shape does
template <typename F>
inline auto with_stencil_shape(int S, int cap, F &&f) {
    if (S == 2) {
        return f.template operator()<2, 1>();
    }
    if (cap <= 2) {
        return f.template operator()<1, 2>();
    }
    return f.template operator()<1, 4>();
}

} // namespace mkb
