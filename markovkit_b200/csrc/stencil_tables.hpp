// Tables of the pair and single-molecule row forms (pair_rows.cuh), and their host-side build:
// one species of at most two molecules, or two species of at most one each, on a structured
// grid whose voxels share one volume class. Reactions enter through per-sector tables indexed by
// the count tuple of one voxel: nA for one species, 2 nA + nB for two.
#pragma once

#include "generator_row.cuh"

#include <cstdint>
#include <vector>

namespace mkb {

constexpr int kStencilIn = 4; // creation reactions per sector the forms handle

template <typename T>
struct StencilSector {
    int begin = 0;                  // first row of the sector in the level space
    int total[2] = {0, 0};          // molecules per species
    int stride0 = 1;                // mixed-radix weight of species 0's rank (species 1's is 1)
    int fast = 0;                   // the forms serve this sector (else the general kernel)
    int n_in = 0;                   // creation reactions with in-jumps into the sector
    int in_copies[kStencilIn] = {}; // copies reaction k creates in its voxel
    int in_src[kStencilIn] = {};    // first row of its source sector
    T exit0 = T(0), leak0 = T(0);   // reactions firing in empty voxels (all voxels)
    T rexit[4] = {}, rleak[4] = {}; // out of one occupied voxel, by its local count tuple
    T rin[kStencilIn][3] = {};      // in-rate of reaction k into a voxel holding n copies
    // reactions whose in-jumps come from every voxel (the source holds c more copies in a voxel
    // w): on rows of at most one molecule whose sources hold at most two
    int n_heavy = 0;
    int heavy_copies[2] = {};       // c of heavy reaction k
    int heavy_src[2] = {};          // first row of its source sector
    int heavy_ok = 0;               // every heavy reaction of the sector is covered
    int pad = 0;
    T rheavy[2][3] = {};            // its rate when the target holds n copies in w
};

template <typename T>
struct StencilView {
    const StencilSector<T> *sectors = nullptr; // per sector of the level (null: forms unused)
    const T *ddeg = nullptr;                   // [species][V]: D_s * sum_e weight_e / volume
    T da[2][3] = {};                           // D_s * weight / volume of an edge along axis a
    int tstride[2] = {2, 1};                   // local count tuple weights
    int gmax = 1;                              // the largest voxel stride of the grid
    int pad = 0;
};

// The per-sector tables of one level, from its sectors (couplings set) and its FP64 model
// tables; false when the level has no structured grid of one volume class or its shape is not
// one species of cap <= 2 or two of cap 1. Sectors the forms cannot serve get fast = 0.
template <typename T>
bool build_stencil_tables(const std::vector<SectorDesc> &sectors, int S, int cap,
                          const ModelView<double> &mv, const std::vector<double> &rate,
                          const std::vector<double> &deg_coef, std::vector<StencilSector<T>> &out,
                          std::vector<T> &ddeg, StencilView<T> &view) {
    out.clear();
    ddeg.clear();
    const bool shape = (S == 1 && cap <= 2) || (S == 2 && cap <= 1);
    if (!shape || mv.grid_dim == 0 || mv.nvc > 1 || mv.vclass) {
        return false;
    }
    const int V = mv.V;
    ddeg.resize(static_cast<std::size_t>(S) * V);
    for (int s = 0; s < S; ++s) {
        for (int v = 0; v < V; ++v) {
            ddeg[static_cast<std::size_t>(s) * V + v] = static_cast<T>(mv.diff[s] * deg_coef[v]);
        }
        for (int a = 0; a < 3; ++a) {
            view.da[s][a] = static_cast<T>(mv.diff[s] * mv.axis_coef[a]);
        }
    }
    view.tstride[0] = S == 2 ? 2 : 1;
    view.tstride[1] = 1;
    view.gmax = mv.gstride[mv.grid_dim - 1];
    const int R = mv.R;
    auto rate_at = [&](int r, int tuple) {
        return rate[static_cast<std::size_t>(r) * mv.ntuple + tuple];
    };
    for (const SectorDesc &sec : sectors) {
        StencilSector<T> ss;
        ss.begin = static_cast<int>(sec.begin);
        ss.total[0] = sec.total[0];
        ss.total[1] = S == 2 ? sec.total[1] : 0;
        ss.stride0 = S == 2 ? static_cast<int>(sec.stride[0]) : 1;
        ss.fast = 1;
        double exit0 = 0.0, leak0 = 0.0;
        for (int r = 0; r < R; ++r) {
            if ((mv.nonneg_mask >> r) & 1U) {
                const double E = mv.empty_total[r];
                if (sec.dst[r] >= 0) {
                    exit0 += E;
                } else {
                    leak0 += E;
                    if (mv.absorbing) {
                        exit0 += E;
                    }
                }
            }
        }
        ss.exit0 = static_cast<T>(exit0);
        ss.leak0 = static_cast<T>(leak0);
        // out of one voxel holding the local tuple (n0[, n1])
        const int nloc = S == 2 ? 4 : 3;
        for (int loc = 0; loc < nloc; ++loc) {
            const int n[2] = {S == 2 ? loc >> 1 : loc, S == 2 ? (loc & 1) : 0};
            bool fits = true;
            int ti = 0;
            for (int s = 0; s < S; ++s) {
                fits = fits && (R == 0 || n[s] <= mv.tmax[s]);
                ti += n[s] * mv.tstride[s];
            }
            double ex = 0.0, lk = 0.0;
            for (int r = 0; r < R && fits; ++r) {
                bool valid = true;
                for (int s = 0; s < S; ++s) {
                    valid = valid && n[s] + mv.change[r][s] >= 0;
                }
                double a = valid ? rate_at(r, ti) : 0.0;
                if ((mv.nonneg_mask >> r) & 1U) {
                    a -= rate_at(r, 0);
                }
                if (sec.dst[r] >= 0) {
                    ex += a;
                } else {
                    lk += a;
                    if (mv.absorbing) {
                        ex += a;
                    }
                }
            }
            ss.rexit[loc] = static_cast<T>(ex);
            ss.rleak[loc] = static_cast<T>(lk);
        }
        // in-jumps of heavy reactions: one species, c = -change copies more in the source, the
        // source holding at most two molecules
        ss.heavy_ok = 1;
        for (int r = 0; r < R; ++r) {
            if (!((mv.heavy_mask >> r) & 1U) || sec.src[r] < 0) {
                continue;
            }
            const int c = -mv.change[r][0];
            if (S != 1 || c < 1 || sec.total[0] + c > 2 || ss.n_heavy >= 2) {
                ss.heavy_ok = 0;
                continue;
            }
            const int k = ss.n_heavy++;
            ss.heavy_copies[k] = c;
            ss.heavy_src[k] = static_cast<int>(sectors[sec.src[r]].begin);
            for (int nv = 0; nv <= 2; ++nv) {
                const int m = nv + c;
                const double a = m <= mv.tmax[0] ? rate_at(r, m) : 0.0;
                ss.rheavy[k][nv] = static_cast<T>(a > 0.0 ? a : 0.0);
            }
        }
        // in-jumps of light reactions: creations of one species only
        for (int r = 0; r < R; ++r) {
            if (((mv.heavy_mask >> r) & 1U) || sec.src[r] < 0) {
                continue;
            }
            const int c = mv.change[r][0];
            if (S != 1 || c < 1 || c > 2 || ss.n_in >= kStencilIn) {
                ss.fast = 0;
                continue;
            }
            const int k = ss.n_in++;
            ss.in_copies[k] = c;
            ss.in_src[k] = static_cast<int>(sectors[sec.src[r]].begin);
            for (int nv = 0; nv <= 2; ++nv) {
                const int m = nv - c;
                const double a = (m >= 0 && m <= mv.tmax[0]) ? rate_at(r, m) : 0.0;
                ss.rin[k][nv] = static_cast<T>(a > 0.0 ? a : 0.0);
            }
        }
        out.push_back(ss);
    }
    return true;
}

} // namespace mkb
