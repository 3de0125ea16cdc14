// One row of the RDME generator, matrix-free: the exit rate, leak rate and every in-jump of
// a state, computed from its unranked molecule lists. Shared by the sm_100a kernels (gather
// SpMV, residuals, smoothers) and by host set-up (dense terminal blocks) and the tests' CPU
// emulation.
//
// Semantics follow markovkit/rdme/reaction_diffusion.hpp:82-118 and generator.hpp:27-44:
//  * a molecule of species s jumps from voxel v along edge e at rate n * D_s * w_e / vol_v;
//  * a local reaction fires in voxel v at rate(counts_v, vol_v) when that rate is positive
//    and the result has no negative count; rates are tabulated per (reaction, volume class,
//    count tuple) on the host, because the reference's rates are host callables;
//  * a jump whose result is outside the space adds to leak, and also to exit when the
//    generator is absorbing.
// The reference scatters each column (generator.hpp:62-81); this gathers each row, so
//   (s I - Q x)_i = (s + exit_i) x_i - sum_{j -> i} rate_{j->i} x_j.
// In-jumps of reactions whose source can sit in any empty voxel (deaths, annihilations)
// fan in from all V voxels; those rows are split across a warp's or a block's threads
// ("heavy" rows).
//
// NS (species) and TMAX (molecules of one species) are compile-time bounds of the state's
// molecule lists; species s < NS with s >= S carry no molecules.
#pragma once

#include "population_index.cuh"

#include <cmath>

namespace mkb {

template <typename T>
struct ModelView {
    int V = 0, S = 0, R = 0;
    int absorbing = 1;
    const int *nbr_ptr = nullptr;            // V + 1
    const int *nbr_idx = nullptr;            // E
    const T *in_coef = nullptr;              // E: weight(w -> v) / vol_w for the edge (v, w)
    const T *deg_coef = nullptr;             // V: sum_e weight(v -> e) / vol_v
    const unsigned char *vparity = nullptr;  // V: checkerboard colour of each voxel (grids)
    const int *vclass = nullptr;             // V: volume class, null when all volumes agree
    const T *rate = nullptr;                 // [R][nvc][ntuple]
    T diff[kMaxSpecies] = {};
    T empty_total[kMaxReactions] = {};       // sum over voxels of the rate out of an empty voxel
    int change[kMaxReactions][kMaxSpecies] = {};
    int tmax[kMaxSpecies] = {};
    int tstride[kMaxSpecies] = {};
    int ntuple = 1;
    int nvc = 1;
    unsigned heavy_mask = 0;  // reactions with in-jumps from empty voxels
    unsigned nonneg_mask = 0; // reactions that can fire from an empty voxel
    // structured grid with one cell volume: neighbours and coefficients by arithmetic
    int grid_dim = 0;         // 0: use the CSR lists above
    int gdims[3] = {1, 1, 1};
    int gstride[3] = {1, 1, 1};
    float ginv[3] = {1, 1, 1}; // 1 / gdims for coordinate division
    T axis_coef[3] = {};       // weight / volume of an edge along each axis
    int stencil = 0;           // grid model without reactions: one-molecule rows are a stencil
    // structured grid: per voxel, bit 2a (2a + 1) set when it has a lower (upper) neighbour
    // along axis a, bit 6 its checkerboard colour (null for general graphs)
    const unsigned *vmask = nullptr;
};

constexpr unsigned kVoxelColourBit = 6;

// q = v / d for 0 <= v < 2^24 from a float reciprocal and one correction
MK_HD int div_small(int v, int d, float inv) {
    int q = static_cast<int>(static_cast<float>(v) * inv);
    q -= (q * d > v) ? 1 : 0;
    q += ((q + 1) * d <= v) ? 1 : 0;
    return q;
}

// coordinates of voxel v on a structured grid (axis 0 fastest)
template <typename T>
MK_HD void grid_coords(const ModelView<T> &md, int v, int (&c)[3]) {
    const int q0 = div_small(v, md.gdims[0], md.ginv[0]);
    c[0] = v - q0 * md.gdims[0];
    const int q1 = div_small(q0, md.gdims[1], md.ginv[1]);
    c[1] = q0 - q1 * md.gdims[1];
    c[2] = q1;
}

template <typename T>
MK_HD T load_ro(const T *p) {
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

// The compiled state shapes: (species S, largest species total `cap`) -> (NS, TMAX); calls
// f.template operator()<NS, TMAX>(). Shared by the kernel launches and the CPU emulation so
// both run the same instantiation.
template <typename F>
inline auto with_shape(int S, int cap, F &&f) {
    if (S == 1) {
        if (cap <= 2) {
            return f.template operator()<1, 2>();
        }
        if (cap <= 4) {
            return f.template operator()<1, 4>();
        }
        if (cap <= 16) {
            return f.template operator()<1, 16>();
        }
        return f.template operator()<1, 64>();
    }
    if (S == 2) {
        if (cap <= 1) {
            return f.template operator()<2, 1>();
        }
        if (cap <= 2) {
            return f.template operator()<2, 2>();
        }
        if (cap <= 4) {
            return f.template operator()<2, 4>();
        }
        return f.template operator()<2, 16>();
    }
    if (cap <= 4) {
        return f.template operator()<kMaxSpecies, 4>();
    }
    return f.template operator()<kMaxSpecies, 16>();
}

// the unranked state of one row: species s's molecules u[s][0..total_s), ascending.
// Index arithmetic inside a level space is 32-bit: level spaces hold fewer than 2^31 states.
template <int NS, int TMAX>
struct RowState {
    int u[NS][TMAX];
    int rank[NS]; // per-species rank inside the sector
};

template <int NS>
MK_HD void split_species(const SectorDesc &sec, int S, std::int64_t local, int (&rank)[NS]) {
    int rem = static_cast<int>(local);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (s + 1 >= S) {
            rank[s] = s + 1 == S ? rem : 0;
        } else {
            const int stride = static_cast<int>(sec.stride[s]);
            int q = static_cast<int>(static_cast<double>(rem) * sec.inv_stride[s]);
            q -= (q * stride > rem) ? 1 : 0;
            q += ((q + 1) * stride <= rem) ? 1 : 0;
            rank[s] = q;
            rem -= q * stride;
        }
    }
}

template <int NS, int TMAX>
MK_HD void load_state(const BinomTable &B, const SectorDesc &sec, int S, int V, std::int64_t local,
                      RowState<NS, TMAX> &st) {
    split_species<NS>(sec, S, local, st.rank);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        unrank_species<TMAX>(B, st.rank[s], s < S ? sec.total[s] : 0, V, st.u[s]);
    }
}

// checkerboard colour of a state: parity of the sum over molecules of their voxel's colour
template <typename T, int NS, int TMAX>
MK_HD int state_colour(const ModelView<T> &md, const SectorDesc &sec, const RowState<NS, TMAX> &st) {
    int c = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        MK_UNROLL_MOL
        for (int p = 0; p < TMAX; ++p) {
            if (p < sec.total[s]) {
                c ^= md.vparity[md.V - 1 - st.u[s][p]];
            }
        }
    }
    return c;
}

// global index of the source state of reaction r's in-jump at voxel uu (source sector ss)
template <typename T, int NS, int TMAX>
MK_HD int reaction_source(const BinomTable &B, const ModelView<T> &md, const SectorDesc &sec,
                          const SectorDesc &ss, const RowState<NS, TMAX> &st, int r, int uu) {
    int src = static_cast<int>(ss.begin);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int c = md.change[r][s];
        const int rs = c == 0 ? st.rank[s]
                              : static_cast<int>(rank_modified<TMAX>(B, st.u[s], sec.total[s],
                                                                     uu, -c));
        src += rs * static_cast<int>(ss.stride[s]);
    }
    return src;
}

// Diffusion of species s: each molecule's exit rate, and the in-jumps into its voxel from each
// neighbour w (the source state has one molecule of that voxel moved to w). A run of equal
// molecules is entered once per neighbour: from above through its last copy, from below
// through its first. When the moved molecule keeps its place in the sorted list, the source
// rank differs by C(u' + p, p + 1) - C(u + p, p + 1) for its position p; only a move past a
// neighbouring molecule re-ranks the whole list (lists of up to two use a closed form).
// On a structured grid the neighbours and edge coefficients are arithmetic, not loaded.
template <typename T, int NS, int TMAX, bool WANT_IN, bool WANT_REV, typename Acc>
MK_HD void diffusion_terms(const BinomTable &B, const ModelView<T> &md, const SectorDesc &sec,
                           const RowState<NS, TMAX> &st, int s, int row, T &exit, Acc &acc) {
    const int t = sec.total[s];
    const int V = md.V;
    const T Ds = md.diff[s];
    const int stride = static_cast<int>(sec.stride[s]);
    const int(&u)[TMAX] = st.u[s];
    auto one = [&](auto P) {
        constexpr int p = decltype(P)::value;
        if (p >= t) {
            return;
        }
        const int uu = u[p];
        const int v = V - 1 - uu;
        const bool first = p == 0 || u[p > 0 ? p - 1 : 0] != uu;
        const bool last = p + 1 >= t || u[p + 1 < TMAX ? p + 1 : p] != uu;
        [[maybe_unused]] const int lo = p > 0 ? u[p > 0 ? p - 1 : 0] : -1;
        [[maybe_unused]] const int hi = p + 1 < t ? u[p + 1 < TMAX ? p + 1 : p] : 0x7fffffff;
        [[maybe_unused]] constexpr int J = p + 1 <= 4 ? p + 1 : 4;
        // the in-jump from the neighbour whose reversed index is uw, with edge coefficient coef;
        // the third argument of acc is the reverse jump's rate (one of this voxel's copies
        // moving back), exact on grids of equal cell volumes where coef is symmetric
        auto in_jump = [&](int uw, T coef) {
            const bool up = uw > uu;
            if (up ? !last : !first) {
                return;
            }
            const int nw = count_of<TMAX>(u, t, uw);
            const T rate = T(nw + 1) * Ds * coef;
            T rev = T(0);
            if constexpr (WANT_REV) {
                rev = T(count_of<TMAX>(u, t, uu)) * Ds * coef;
            }
            int delta;
            if constexpr (TMAX <= 2) {
                delta = static_cast<int>(rank_replace<TMAX>(B, u, t, uu, uw)) - st.rank[s];
            } else if (up ? uw <= hi : uw >= lo) {
                delta = static_cast<int>(binom_j<J>(uw + p) - binom_j<J>(uu + p));
            } else {
                delta = static_cast<int>(rank_replace<TMAX>(B, u, t, uu, uw)) - st.rank[s];
            }
            acc(row + delta * stride, rate, rev);
        };
        if (md.grid_dim > 0) {
            int c[3];
            grid_coords(md, v, c);
            T deg = T(0);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const bool has_lo = c[a] > 0, has_hi = c[a] + 1 < md.gdims[a];
                deg += T((has_lo ? 1 : 0) + (has_hi ? 1 : 0)) * md.axis_coef[a];
                if constexpr (WANT_IN) {
                    // neighbour v - stride has reversed index uu + stride, v + stride uu - stride
                    if (has_lo && (first || last)) {
                        in_jump(uu + md.gstride[a], md.axis_coef[a]);
                    }
                    if (has_hi && (first || last)) {
                        in_jump(uu - md.gstride[a], md.axis_coef[a]);
                    }
                }
            }
            exit += Ds * deg;
            return;
        }
        exit += Ds * load_ro(md.deg_coef + v);
        if constexpr (WANT_IN) {
            if (!first && !last) {
                return;
            }
            const int e0 = load_ro(md.nbr_ptr + v), e1 = load_ro(md.nbr_ptr + v + 1);
            for (int e = e0; e < e1; ++e) {
                in_jump(V - 1 - load_ro(md.nbr_idx + e), load_ro(md.in_coef + e));
            }
        }
    };
    if constexpr (TMAX <= 4) {
        static_for<TMAX>(one);
    } else {
        // long lists: a plain loop over the CSR lists, re-ranking every in-jump
        for (int p = 0; p < t; ++p) {
            const int uu = u[p];
            const int v = V - 1 - uu;
            exit += Ds * load_ro(md.deg_coef + v);
            if constexpr (WANT_IN) {
                const bool first = p == 0 || u[p - 1] != uu;
                const bool last = p + 1 >= t || u[p + 1] != uu;
                const int e0 = load_ro(md.nbr_ptr + v), e1 = load_ro(md.nbr_ptr + v + 1);
                for (int e = e0; e < e1; ++e) {
                    const int uw = V - 1 - load_ro(md.nbr_idx + e);
                    if (uw > uu ? !last : !first) {
                        continue;
                    }
                    const int nw = count_of<TMAX>(u, t, uw);
                    const T rate = T(nw + 1) * Ds * load_ro(md.in_coef + e);
                    const int delta =
                        static_cast<int>(rank_replace<TMAX>(B, u, t, uu, uw)) - st.rank[s];
                    T rev = T(0);
                    if constexpr (WANT_REV) {
                        rev = T(count_of<TMAX>(u, t, uu)) * Ds * load_ro(md.in_coef + e);
                    }
                    acc(row + delta * stride, rate, rev);
                }
            }
        }
    }
}

// rank of the list with one more copy of `value`: an element left of the insertion point keeps
// its position (A_i = C(u_i + i, i + 1)), one right of it moves up one (B_i = C(u_i + i + 1,
// i + 2)); the new element lands after the b smaller ones. A and B are per-row constants.
template <int TMAX>
MK_HD std::int64_t rank_inserted(const int (&u)[TMAX], int t, const std::int64_t (&A)[TMAX],
                                 const std::int64_t (&Bc)[TMAX], int value) {
    std::int64_t r = 0;
    int b = 0;
#pragma unroll
    for (int i = 0; i < TMAX; ++i) {
        if (i < t) {
            const bool left = u[i] < value;
            r += left ? A[i] : Bc[i];
            b += left ? 1 : 0;
        }
    }
    std::int64_t mine = 0;
    static_for<TMAX + 1>([&](auto Q) {
        constexpr int q = decltype(Q)::value;
        constexpr int J = q + 1 <= 4 ? q + 1 : 4;
        mine = b == q ? binom_j<J>(value + q) : mine;
    });
    return r + mine;
}

// A row of a diffusion-only model on a structured grid whose species hold at most one molecule
// each (TMAX 1): the state is one voxel per present species, and each in-jump moves one of them
// in from a grid neighbour, so its source index is row + (uw - uu) * stride_s with
// uw = uu +/- gstride. The terms, their values and their order are those of diffusion_terms
// (rate = 1 * D_s * coef, the lower neighbour first), so the results are bit-identical; what
// goes is the general machinery (run detection, counts, re-ranking) around them.
template <typename T, int NS, bool WANT_IN, bool WANT_REV, typename Acc>
MK_HD void stencil_row(const ModelView<T> &md, const SectorDesc &sec, const RowState<NS, 1> &st,
                       int row, T &exit, Acc &acc) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (sec.total[s] < 1) {
            continue;
        }
        const T Ds = md.diff[s];
        const int stride = static_cast<int>(sec.stride[s]);
        int c[3];
        grid_coords(md, md.V - 1 - st.u[s][0], c);
        T deg = T(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a >= md.grid_dim) {
                continue;
            }
            const bool has_lo = c[a] > 0, has_hi = c[a] + 1 < md.gdims[a];
            deg += T((has_lo ? 1 : 0) + (has_hi ? 1 : 0)) * md.axis_coef[a];
            if constexpr (WANT_IN) {
                const T rate = T(1) * Ds * md.axis_coef[a];
                const T rev = WANT_REV ? rate : T(0);
                const int step = md.gstride[a] * stride;
                if (has_lo) {
                    acc(row + step, rate, rev);
                }
                if (has_hi) {
                    acc(row - step, rate, rev);
                }
            }
        }
        exit += Ds * deg;
    }
}

// Reactions that fire from empty voxels: their all-empty total goes to exit (or leak when the
// product leaves the space); light rows only.
template <typename T>
MK_HD void empty_reaction_terms(const SectorDesc &sec, const ModelView<T> &md, T &exit, T &leak) {
    for (int r = 0; r < md.R; ++r) {
        if (!((md.nonneg_mask >> r) & 1U)) {
            continue;
        }
        const T E = md.empty_total[r];
        if (sec.dst[r] >= 0) {
            exit += E;
        } else {
            leak += E;
            if (md.absorbing) {
                exit += E;
            }
        }
    }
}

// Local reactions of the occupied voxels, each distinct voxel once at the first occurrence
// (s, p) of it: the rate out of the voxel (corrected for the all-empty total counted above),
// and the in-jumps of reactions whose source is a state with the voxel's counts changed
// (heavy reactions, whose sources can sit in any empty voxel, are visited separately).
template <typename T, int NS, int TMAX, bool WANT_IN, typename Acc>
MK_HD void occupied_reaction_terms(const BinomTable &B, const SectorDesc *sectors,
                                   const SectorDesc &sec, const ModelView<T> &md,
                                   const RowState<NS, TMAX> &st, T &exit, T &leak, Acc &acc) {
    const int V = md.V, R = md.R;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        MK_UNROLL_MOL
        for (int p = 0; p < TMAX; ++p) {
            if (R == 0 || p >= sec.total[s]) {
                continue;
            }
            const int uu = st.u[s][p];
            if (p > 0 && st.u[s][p - 1] == uu) {
                continue;
            }
            bool seen = false;
#pragma unroll
            for (int s2 = 0; s2 < s; ++s2) {
                seen = seen || count_of<TMAX>(st.u[s2], sec.total[s2], uu) > 0;
            }
            if (seen) {
                continue;
            }
            const int v = V - 1 - uu;
            int n[NS];
            int ti = 0;
#pragma unroll
            for (int s2 = 0; s2 < NS; ++s2) {
                n[s2] = count_of<TMAX>(st.u[s2], sec.total[s2], uu);
                ti += n[s2] * md.tstride[s2];
            }
            const int vc = md.vclass ? load_ro(md.vclass + v) : 0;
            for (int r = 0; r < R; ++r) {
                const T *rrow = md.rate + (static_cast<std::int64_t>(r) * md.nvc + vc) * md.ntuple;
                bool valid = true;
                int tm = 0;
                bool ok = true;
#pragma unroll
                for (int s4 = 0; s4 < NS; ++s4) {
                    valid = valid && n[s4] + md.change[r][s4] >= 0;
                    const int m = n[s4] - md.change[r][s4];
                    ok = ok && m >= 0 && m <= md.tmax[s4];
                    tm += m * md.tstride[s4];
                }
                // out of this voxel; and it is not one of the empty voxels counted above
                T a = valid ? load_ro(rrow + ti) : T(0);
                if ((md.nonneg_mask >> r) & 1U) {
                    a -= load_ro(rrow);
                }
                if (sec.dst[r] >= 0) {
                    exit += a;
                } else {
                    leak += a;
                    if (md.absorbing) {
                        exit += a;
                    }
                }
                if constexpr (WANT_IN) {
                    if (((md.heavy_mask >> r) & 1U) || sec.src[r] < 0 || !ok) {
                        continue;
                    }
                    const T ain = load_ro(rrow + tm);
                    if (ain > T(0)) {
                        acc(reaction_source<T, NS, TMAX>(B, md, sec, sectors[sec.src[r]], st, r, uu),
                            ain, T(0));
                    }
                }
            }
        }
    }
}

// Visit the row: acc(source_index, rate) for every in-jump; adds into exit and leak.
// light: the exit/leak terms and the in-jumps that start in occupied voxels.
// [lane, V) step nlanes: the all-voxel loop of heavy reactions.
template <typename T, int NS, int TMAX, bool WANT_IN = true, bool WANT_REV = false, typename Acc>
MK_HD void visit_row(const BinomTable &B, const SectorDesc *sectors, const SectorDesc &sec,
                     const ModelView<T> &md, std::int64_t local, const RowState<NS, TMAX> &st,
                     bool light, int lane, int nlanes, T &exit, T &leak, Acc &&acc) {
    const int V = md.V, R = md.R;
    if constexpr (TMAX == 1) {
        if (md.stencil && light && nlanes == 1) {
            stencil_row<T, NS, WANT_IN, WANT_REV>(md, sec, st, static_cast<int>(sec.begin + local),
                                                  exit, acc);
            return;
        }
    }
    if (light) {
        empty_reaction_terms<T>(sec, md, exit, leak);
        // diffusion, molecule by molecule: out of its voxel, and into it from each neighbour
        const int row = static_cast<int>(sec.begin + local);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            diffusion_terms<T, NS, TMAX, WANT_IN, WANT_REV>(B, md, sec, st, s, row, exit, acc);
        }
        occupied_reaction_terms<T, NS, TMAX, WANT_IN>(B, sectors, sec, md, st, exit, leak, acc);
    }
    // heavy reactions: a source in every voxel
    if constexpr (WANT_IN) {
        for (int r = 0; r < R; ++r) {
            if (!((md.heavy_mask >> r) & 1U) || sec.src[r] < 0) {
                continue;
            }
            const SectorDesc &ss = sectors[sec.src[r]];
            // the source gains |change| molecules in the visited voxel; species with one more
            // molecule use per-row insertion coefficients (lists of up to three, or of four
            // with one species: the source then holds at most four, as a list of four has no
            // source sector), others the general re-rank
            constexpr bool kInsert = TMAX <= 3 || (TMAX == 4 && NS == 1);
            std::int64_t A[NS][TMAX], Bc[NS][TMAX];
            int fixed = static_cast<int>(ss.begin);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                if (md.change[r][s] == 0) {
                    fixed += st.rank[s] * static_cast<int>(ss.stride[s]);
                }
                if constexpr (kInsert) {
                    static_for<TMAX>([&](auto I) {
                        constexpr int i = decltype(I)::value;
                        A[s][i] = binom_j<i + 1>(st.u[s][i] + i);
                        // molecule i moves up a place only when i < t <= 3
                        if constexpr (i + 2 <= 4) {
                            Bc[s][i] = binom_j<i + 2>(st.u[s][i] + i + 1);
                        } else {
                            Bc[s][i] = 0;
                        }
                    });
                }
            }
            // unrolled so that several lanes' gathers are in flight at once
#pragma unroll 4
            for (int v = lane; v < V; v += nlanes) {
                const int uu = V - 1 - v;
                int tm = 0;
                bool ok = true;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const int m = count_of<TMAX>(st.u[s], sec.total[s], uu) - md.change[r][s];
                    ok = ok && m >= 0 && m <= md.tmax[s];
                    tm += m * md.tstride[s];
                }
                if (!ok) {
                    continue;
                }
                const int vc = md.vclass ? load_ro(md.vclass + v) : 0;
                const T a = load_ro(md.rate +
                                    (static_cast<std::int64_t>(r) * md.nvc + vc) * md.ntuple + tm);
                if (!(a > T(0))) {
                    continue;
                }
                int src = fixed;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const int c = md.change[r][s];
                    if (c == 0) {
                        continue;
                    }
                    std::int64_t rs;
                    if constexpr (kInsert) {
                        rs = c == -1 && sec.total[s] < 4
                                 ? rank_inserted<TMAX>(st.u[s], sec.total[s], A[s], Bc[s], uu)
                                     : rank_modified<TMAX>(B, st.u[s], sec.total[s], uu, -c);
                    } else {
                        rs = rank_modified<TMAX>(B, st.u[s], sec.total[s], uu, -c);
                    }
                    src += static_cast<int>(rs) * static_cast<int>(ss.stride[s]);
                }
                acc(src, a, T(0));
            }
        }
    }
}

// Multigrid transfer between the same sector on a fine and a coarse grid
// (markovkit/rdme/multigrid.hpp:48-111): each fine state maps to the coarse state with the
// same count in every coarse voxel, with the multinomial weight
//   w = prod_a [c_a! / prod_{v in a} n_v!] * children_a^{-c_a}.
// Those weights sum to one over the fine states of a coarse state exactly, so the
// reference's renormalisation (:89-91) only removes rounding and is not repeated here.
struct TransferView {
    int Vc = 0;
    const int *parent = nullptr;          // fine voxel -> coarse voxel
    const double *log_children = nullptr; // per coarse voxel
    const double *lgf = nullptr;          // log(k!) for k = 0..kmax
    const SectorDesc *coarse_sectors = nullptr;
};

// the coarse index of a fine state and (optionally) its prolongation weight; the coarse
// molecule list is ranked without sorting: an element of value w at sorted position q adds
// C(w + q, q + 1), q = (#smaller) + (#equal ones before it)
template <int NS, int TMAX>
MK_HD std::int64_t coarse_index(const BinomTable &B, const TransferView &tv, const SectorDesc &fine,
                                int Vf, const RowState<NS, TMAX> &st, double *weight) {
    const SectorDesc &cs = tv.coarse_sectors[fine.coarse];
    std::int64_t index = cs.begin;
    double logw = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int t = fine.total[s];
        int cu[TMAX];
        MK_UNROLL_MOL
        for (int p = 0; p < TMAX; ++p) {
            cu[p] = p < t ? tv.Vc - 1 - load_ro(tv.parent + (Vf - 1 - st.u[s][p])) : 0;
        }
        std::int64_t r = 0;
        MK_UNROLL_MOL
        for (int p = 0; p < TMAX; ++p) {
            if (p >= t) {
                continue;
            }
            int q = 0, equal_before = 0, equal_total = 0;
            MK_UNROLL_MOL
            for (int k = 0; k < TMAX; ++k) {
                if (k < t) {
                    q += cu[k] < cu[p] ? 1 : 0;
                    equal_before += (k < p && cu[k] == cu[p]) ? 1 : 0;
                    equal_total += cu[k] == cu[p] ? 1 : 0;
                }
            }
            q += equal_before;
            r += binom(B, cu[p] + q, q + 1);
            if (weight) {
                if (equal_before == 0) {
                    // first copy of a coarse value: lgamma(c_a + 1) - c_a log(children_a)
                    logw += load_ro(tv.lgf + equal_total) -
                            equal_total * load_ro(tv.log_children + (tv.Vc - 1 - cu[p]));
                }
                if (p == 0 || st.u[s][p - 1] != st.u[s][p]) {
                    // first copy of a fine value: - lgamma(n_v + 1)
                    logw -= load_ro(tv.lgf + count_of<TMAX>(st.u[s], t, st.u[s][p]));
                }
            }
        }
        index += r * cs.stride[s];
    }
    if (weight) {
        *weight = std::exp(logw);
    }
    return index;
}

} // namespace mkb
