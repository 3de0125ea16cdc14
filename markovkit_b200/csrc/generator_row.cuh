// One row of the RDME generator, matrix-free: the exit rate, leak rate and every in-jump of
// a state, computed from its unranked molecule lists. Shared by the sm_100a kernels (gather
// SpMV, residuals, smoothers) and by host set-up (dense terminal blocks).
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
// fan in from all V voxels; those rows are split across a warp's lanes ("heavy" rows).
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
};

template <typename T>
MK_HD T load_ro(const T *p) {
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

template <typename T>
MK_HD int load_ro_i(const int *p) {
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

// the unranked state of one row
template <int MAXM>
struct RowState {
    int u[MAXM];                       // molecule lists, species-major, ascending per species
    std::int64_t rank[kMaxSpecies];    // per-species rank inside the sector
};

template <int MAXM>
MK_HD void load_state(const BinomTable &B, const SectorDesc &sec, int S, int V, std::int64_t local,
                      RowState<MAXM> &st) {
    split_local(sec, S, local, st.rank);
    for (int s = 0; s < S; ++s) {
        unrank_species(B, st.rank[s], sec.total[s], V, st.u + sec.mol_offset[s]);
    }
}

// checkerboard colour of a state: parity of the sum over molecules of their voxel's colour
template <typename T, int MAXM>
MK_HD int state_colour(const ModelView<T> &md, const SectorDesc &sec, const RowState<MAXM> &st) {
    int c = 0;
    for (int p = 0; p < sec.n_mol; ++p) {
        c ^= md.vparity[md.V - 1 - st.u[p]];
    }
    return c;
}

// Visit the row: acc(source_index, rate) for every in-jump; adds into exit and leak.
// light: the exit/leak terms and the in-jumps that start in occupied voxels.
// [lane, V) step nlanes: the all-voxel loop of heavy reactions.
template <typename T, int MAXM, bool WANT_IN = true, typename Acc>
MK_HD void visit_row(const BinomTable &B, const SectorDesc *sectors, const SectorDesc &sec,
                     const ModelView<T> &md, std::int64_t local, const RowState<MAXM> &st,
                     bool light, int lane, int nlanes, T &exit, T &leak, Acc &&acc) {
    const int V = md.V, S = md.S, R = md.R;
    if (light) {
        // distinct occupied voxels across species, ascending in u
        int d[MAXM];
        int nd = 0;
        for (int p = 0; p < sec.n_mol; ++p) {
            const int val = st.u[p];
            int pos = nd;
            bool seen = false;
            for (int q = 0; q < nd; ++q) {
                if (d[q] == val) {
                    seen = true;
                    break;
                }
            }
            if (seen) {
                continue;
            }
            while (pos > 0 && d[pos - 1] > val) {
                d[pos] = d[pos - 1];
                --pos;
            }
            d[pos] = val;
            ++nd;
        }
        T esub[kMaxReactions];
        for (int r = 0; r < R; ++r) {
            esub[r] = T(0);
        }
        for (int q = 0; q < nd; ++q) {
            const int uu = d[q];
            const int v = V - 1 - uu;
            int n[kMaxSpecies];
            int ti = 0;
            for (int s = 0; s < S; ++s) {
                n[s] = count_of(st.u + sec.mol_offset[s], sec.total[s], uu);
                ti += n[s] * md.tstride[s];
            }
            // diffusion: out of v, and into v from each neighbour
            const int e0 = load_ro_i<int>(md.nbr_ptr + v), e1 = load_ro_i<int>(md.nbr_ptr + v + 1);
            for (int s = 0; s < S; ++s) {
                if (n[s] == 0) {
                    continue;
                }
                const int *us = st.u + sec.mol_offset[s];
                const int ts = sec.total[s];
                exit += T(n[s]) * md.diff[s] * load_ro(md.deg_coef + v);
                if (!WANT_IN) {
                    continue;
                }
                for (int e = e0; e < e1; ++e) {
                    const int w = load_ro_i<int>(md.nbr_idx + e);
                    const int uw = V - 1 - w;
                    const int nw = count_of(us, ts, uw);
                    const T rate = T(nw + 1) * md.diff[s] * load_ro(md.in_coef + e);
                    const std::int64_t r2 = rank_replace(B, us, ts, uu, uw);
                    acc(sec.begin + local + (r2 - st.rank[s]) * sec.stride[s], rate);
                }
            }
            if (R == 0) {
                continue;
            }
            const int vc = md.vclass ? load_ro_i<int>(md.vclass + v) : 0;
            for (int r = 0; r < R; ++r) {
                const T *rrow = md.rate + (static_cast<std::int64_t>(r) * md.nvc + vc) * md.ntuple;
                bool valid = true;
                for (int s = 0; s < S; ++s) {
                    valid = valid && (n[s] + md.change[r][s] >= 0);
                }
                if (valid) {
                    const T a = load_ro(rrow + ti);
                    if (a > T(0)) {
                        if (sec.dst[r] >= 0) {
                            exit += a;
                        } else {
                            leak += a;
                            if (md.absorbing) {
                                exit += a;
                            }
                        }
                    }
                }
                if ((md.nonneg_mask >> r) & 1U) {
                    const T a0 = load_ro(rrow);
                    esub[r] += a0 > T(0) ? a0 : T(0);
                }
                if (!WANT_IN || ((md.heavy_mask >> r) & 1U) || sec.src[r] < 0) {
                    continue;
                }
                int tm = 0;
                bool ok = true;
                for (int s = 0; s < S; ++s) {
                    const int m = n[s] - md.change[r][s];
                    ok = ok && m >= 0 && m <= md.tmax[s];
                    tm += m * md.tstride[s];
                }
                if (!ok) {
                    continue;
                }
                const T a = load_ro(rrow + tm);
                if (!(a > T(0))) {
                    continue;
                }
                const SectorDesc &ss = sectors[sec.src[r]];
                std::int64_t src = ss.begin;
                for (int s = 0; s < S; ++s) {
                    const std::int64_t rs =
                        md.change[r][s] == 0
                            ? st.rank[s]
                            : rank_modified(B, st.u + sec.mol_offset[s], sec.total[s], uu,
                                            -md.change[r][s]);
                    src += rs * ss.stride[s];
                }
                acc(src, a);
            }
        }
        // reactions that fire from the empty voxels: the all-empty total minus occupied voxels
        for (int r = 0; r < R; ++r) {
            if (!((md.nonneg_mask >> r) & 1U)) {
                continue;
            }
            const T E = md.empty_total[r] - esub[r];
            if (!(E > T(0))) {
                continue;
            }
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
    // heavy reactions: a source in every voxel
    if (!WANT_IN) {
        return;
    }
    for (int r = 0; r < R; ++r) {
        if (!((md.heavy_mask >> r) & 1U) || sec.src[r] < 0) {
            continue;
        }
        const SectorDesc &ss = sectors[sec.src[r]];
        for (int v = lane; v < V; v += nlanes) {
            const int uu = V - 1 - v;
            int tm = 0;
            bool ok = true;
            for (int s = 0; s < S; ++s) {
                const int m =
                    count_of(st.u + sec.mol_offset[s], sec.total[s], uu) - md.change[r][s];
                ok = ok && m >= 0 && m <= md.tmax[s];
                tm += m * md.tstride[s];
            }
            if (!ok) {
                continue;
            }
            const int vc = md.vclass ? load_ro_i<int>(md.vclass + v) : 0;
            const T a =
                load_ro(md.rate + (static_cast<std::int64_t>(r) * md.nvc + vc) * md.ntuple + tm);
            if (!(a > T(0))) {
                continue;
            }
            std::int64_t src = ss.begin;
            for (int s = 0; s < S; ++s) {
                const std::int64_t rs =
                    md.change[r][s] == 0
                        ? st.rank[s]
                        : rank_modified(B, st.u + sec.mol_offset[s], sec.total[s], uu,
                                        -md.change[r][s]);
                src += rs * ss.stride[s];
            }
            acc(src, a);
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

// the coarse index of a fine state and (optionally) its prolongation weight
template <int MAXM>
MK_HD std::int64_t coarse_index(const BinomTable &B, const TransferView &tv, const SectorDesc &fine,
                                int S, int Vf, const RowState<MAXM> &st, double *weight) {
    const SectorDesc &cs = tv.coarse_sectors[fine.coarse];
    std::int64_t index = cs.begin;
    double logw = 0.0;
    for (int s = 0; s < S; ++s) {
        const int t = fine.total[s];
        const int *u = st.u + fine.mol_offset[s];
        int cu[MAXM];
        for (int p = 0; p < t; ++p) {
            const int a = load_ro_i<int>(tv.parent + (Vf - 1 - u[p]));
            int val = tv.Vc - 1 - a;
            int pos = p;
            while (pos > 0 && cu[pos - 1] > val) {
                cu[pos] = cu[pos - 1];
                --pos;
            }
            cu[pos] = val;
        }
        index += rank_species(B, cu, t) * cs.stride[s];
        if (weight) {
            for (int p = 0; p < t;) {
                int q = p;
                while (q < t && u[q] == u[p]) {
                    ++q;
                }
                logw -= load_ro(tv.lgf + (q - p));
                p = q;
            }
            for (int p = 0; p < t;) {
                int q = p;
                while (q < t && cu[q] == cu[p]) {
                    ++q;
                }
                const int a = tv.Vc - 1 - cu[p];
                logw += load_ro(tv.lgf + (q - p)) - (q - p) * load_ro(tv.log_children + a);
                p = q;
            }
        }
    }
    if (weight) {
        *weight = exp(logw);
    }
    return index;
}

} // namespace mkb
