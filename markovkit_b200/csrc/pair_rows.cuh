// Rows of the two state shapes the solve workloads live on, on structured grids: one species of
// at most two molecules (a box or sector of cap 2: the 3-D 16^3 box and its multigrid levels),
// and two species of at most one molecule each (the two-particle annihilation box). They visit
// the same in-jumps with the same rates as visit_row (generator_row.cuh), and reach them in few
// instructions:
//  * a pair u0 <= u1 (u = V - 1 - voxel) has rank u0 + T(u1), T(k) = k (k + 1) / 2, so it is
//    unranked by one single-precision square root and an exact correction;
//  * a molecule moving by +-g along an axis changes the rank by +-g (the lower one) or by
//    T(u1 +- g) - T(u1) = +-g u1 + T(g) or T(g - 1) (the upper one), unless the move reorders or
//    joins the pair, when the source rank is min + T(max) of the new pair;
//  * which neighbours exist comes from a per-voxel mask; a molecule's exit rate is a per-voxel
//    table, reactions a per-sector table by the count tuple of the voxel.
// Exit rates add the same terms as visit_row in another order, so the two kernels agree to
// rounding (about 1e-16 relative), not bit for bit.
#pragma once

#include "generator_row.cuh"
#include "stencil_tables.hpp"

#include <math.h>

namespace mkb {

// T(k) = k (k + 1) / 2 for 0 <= k < 65536 (states of a pair sector number below 2^31)
MK_HD int tri(int k) {
    return static_cast<int>((static_cast<unsigned>(k) * static_cast<unsigned>(k + 1)) >> 1);
}

// the pair (u0 <= u1) of rank r < 2^31
MK_HD void unrank_pair(int r, int &u0, int &u1) {
    const float q = 8.0f * static_cast<float>(r) + 1.0f;
    float root;
#if defined(__CUDA_ARCH__)
    // an approximate root is enough: the integer correction below makes k exact
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(root) : "f"(q));
#else
    root = sqrtf(q);
#endif
    int k = static_cast<int>((root - 1.0f) * 0.5f);
    const auto tri64 = [](int q) { return (static_cast<unsigned long long>(q) * (q + 1)) >> 1; };
    k += tri64(k + 1) <= static_cast<unsigned long long>(r) ? 1 : 0;
    k -= tri64(k) > static_cast<unsigned long long>(r) ? 1 : 0;
    u1 = k;
    u0 = r - tri(k);
}

MK_HD bool has_lower(unsigned mask, int a) { return ((mask >> (2 * a)) & 1U) != 0; }
MK_HD bool has_upper(unsigned mask, int a) { return ((mask >> (2 * a + 1)) & 1U) != 0; }

// One species, t <= 2 molecules (u0 <= u1; u0 alone when t = 1), masks m0 and m1 of their
// voxels. acc(source, rate, on) per candidate in-jump in visit_row's order: the in-jump exists
// when on, and the caller reads the source only then (the sum takes rate * 0 otherwise, so
// that lanes of a warp at different boundaries do not diverge).
template <typename T, bool WANT_IN, typename Acc>
MK_HD void pair_row(const ModelView<T> &md, const StencilView<T> &sv, const StencilSector<T> &ss,
                    int t, int u0, int u1, unsigned m0, unsigned m1, int row, T &exit, T &leak,
                    Acc &&acc) {
    const int V = md.V;
    exit += ss.exit0;
    leak += ss.leak0;
    if (t == 0) {
        return;
    }
    const bool same = t == 2 && u0 == u1;
    // diffusion out, then the reactions of each distinct voxel
    exit += load_ro(sv.ddeg + (V - 1 - u0));
    if (t == 2) {
        exit += load_ro(sv.ddeg + (V - 1 - u1));
        if (same) {
            exit += ss.rexit[2];
            leak += ss.rleak[2];
        } else {
            exit += ss.rexit[1] + ss.rexit[1];
            leak += ss.rleak[1] + ss.rleak[1];
        }
    } else {
        exit += ss.rexit[1];
        leak += ss.rleak[1];
    }
    if constexpr (!WANT_IN) {
        return;
    } else {
        if (t == 1) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const int g = md.gstride[a];
                const T D = sv.da[0][a];
                acc(row + g, D, has_lower(m0, a));
                acc(row - g, D, has_upper(m0, a));
            }
            for (int k = 0; k < ss.n_in; ++k) {
                if (ss.in_copies[k] == 1 && ss.rin[k][1] > T(0)) {
                    acc(ss.in_src[k], ss.rin[k][1], true);
                }
            }
            return;
        }
        // t == 2: molecule 0 (the lower u) first, then molecule 1, as visit_row
        const int tu1 = tri(u1);
        if (u1 - u0 > sv.gmax) {
            // no move can reach or pass the other molecule: every source rank is row + const
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const int g = md.gstride[a];
                const T D = sv.da[0][a];
                acc(row + g, D, has_lower(m0, a));
                acc(row - g, D, has_upper(m0, a));
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const int g = md.gstride[a];
                const T D = sv.da[0][a];
                acc(row + g * u1 + tri(g), D, has_lower(m1, a));
                acc(row - g * u1 + tri(g - 1), D, has_upper(m1, a));
            }
        } else {
            const int base = row - u0 - tu1; // first row of the sector
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const int g = md.gstride[a];
                const T D = sv.da[0][a];
                // molecule 0 from above (its run's last copy) and from below (its first)
                if (has_lower(m0, a) && !same) {
                    const int uw = u0 + g;
                    if (uw <= u1) {
                        acc(base + uw + tu1, uw == u1 ? D + D : D, true);
                    } else {
                        acc(base + u1 + tri(uw), D, true);
                    }
                }
                acc(row - g, D, has_upper(m0, a));
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const int g = md.gstride[a];
                const T D = sv.da[0][a];
                acc(base + u0 + tri(u1 + g), D, has_lower(m1, a));
                if (has_upper(m1, a) && !same) {
                    const int uw = u1 - g;
                    if (uw >= u0) {
                        acc(base + u0 + tri(uw), uw == u0 ? D + D : D, true);
                    } else {
                        acc(base + uw + tri(u0), D, true);
                    }
                }
            }
        }
        // creation reactions: the source lacks the created copies in this voxel
        for (int k = 0; k < ss.n_in; ++k) {
            const int c = ss.in_copies[k];
            if (same) {
                const T a = ss.rin[k][2];
                if (a > T(0)) {
                    acc(ss.in_src[k] + (c == 1 ? u0 : 0), a, true);
                }
            } else if (c == 1) {
                const T a = ss.rin[k][1];
                if (a > T(0)) {
                    acc(ss.in_src[k] + u1, a, true); // voxel of u0 loses its copy: {u1} is left
                    acc(ss.in_src[k] + u0, a, true);
                }
            }
        }
    }
}

// The in-jumps of a row's heavy reactions from the voxels w = lane, lane + nlanes, ... (the row
// holds t <= 1 molecule u; the source holds c more copies of w, at most two molecules): source
// rank w (one molecule), w + T(w) (two in w) or min + T(max) of {u, w}; rate by the row's count
// in w. acc(source, rate, on) per candidate in-jump (on: the rate is positive).
template <typename T, typename Acc>
MK_HD void pair_heavy_terms(const StencilSector<T> &ss, int V, int t, int u, int lane, int nlanes,
                            Acc &&acc) {
    for (int k = 0; k < ss.n_heavy; ++k) {
        const int c = ss.heavy_copies[k];
        const int src = ss.heavy_src[k];
        const T a0 = ss.rheavy[k][0], a1 = ss.rheavy[k][1];
        const int tu = t == 1 ? tri(u) : 0;
#pragma unroll 4
        for (int w = lane; w < V; w += nlanes) {
            int rank;
            T a = a0;
            if (t == 0) {
                rank = c == 1 ? w : w + tri(w);
            } else if (w <= u) {
                rank = w + tu;
                a = w == u ? a1 : a0;
            } else {
                rank = u + tri(w);
            }
            acc(src + rank, a, a > T(0));
        }
    }
}

// Two species of at most one molecule each (uA, uB; present when tA, tB), masks mA, mB.
template <typename T, bool WANT_IN, typename Acc>
MK_HD void singles_row(const ModelView<T> &md, const StencilView<T> &sv,
                       const StencilSector<T> &ss, int uA, int uB, unsigned mA, unsigned mB,
                       int row, T &exit, T &leak, Acc &&acc) {
    const int V = md.V;
    const int tA = ss.total[0], tB = ss.total[1];
    exit += ss.exit0;
    leak += ss.leak0;
    if (tA) {
        exit += load_ro(sv.ddeg + (V - 1 - uA));
    }
    if (tB) {
        exit += load_ro(sv.ddeg + V + (V - 1 - uB));
    }
    const int kA = sv.tstride[0], kB = sv.tstride[1];
    if (tA && tB && uA == uB) {
        exit += ss.rexit[kA + kB];
        leak += ss.rleak[kA + kB];
    } else {
        if (tA) {
            exit += ss.rexit[kA];
            leak += ss.rleak[kA];
        }
        if (tB) {
            exit += ss.rexit[kB];
            leak += ss.rleak[kB];
        }
    }
    if constexpr (WANT_IN) {
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (!(s == 0 ? tA : tB)) {
                continue;
            }
            const unsigned m = s == 0 ? mA : mB;
            const int stride = s == 0 ? ss.stride0 : 1;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (a >= md.grid_dim) {
                    continue;
                }
                const int step = md.gstride[a] * stride;
                const T D = sv.da[s][a];
                acc(row + step, D, has_lower(m, a));
                acc(row - step, D, has_upper(m, a));
            }
        }
    }
}

// the rows the pair and single-molecule forms serve: one species of cap <= 2, or two of cap 1
inline bool pair_shape(int S, int cap) { return (S == 1 && cap <= 2) || (S == 2 && cap <= 1); }

} // namespace mkb
