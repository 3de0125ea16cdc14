// Host-only set-up shared by the engine and the CPU emulation used in the tests: binomial
// tables, sector layout, RDME models (grid or explicit graph), per-precision model tables and
// the reaction couplings between sectors. No CUDA runtime calls here.
#pragma once

#include "generator_row.cuh"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace mkb {

// status codes, shared with the C ABI (include/markovkit_b200.h)
enum Status : int {
    kOk = 0,
    kEInval = 1,
    kEOverflow = 2,
    kESingular = 3,
    kENoMem = 4,
    kENotConv = 5,
    kENan = 6,
    kETimeout = 7,
    kECuda = 8,
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &what) : std::runtime_error(what), code(c) {}
};

constexpr std::int64_t kSaturated = std::int64_t(1) << 62;

// C(q, j) for 0 <= j <= jmax, 0 <= q <= qmax, row-major by j, saturating at 2^62
inline std::vector<std::int64_t> binomial_table(int jmax, int qmax) {
    std::vector<std::int64_t> t(static_cast<std::size_t>(jmax + 1) * (qmax + 1), 0);
    auto at = [&](int j, int q) -> std::int64_t & {
        return t[static_cast<std::size_t>(j) * (qmax + 1) + q];
    };
    for (int q = 0; q <= qmax; ++q) {
        at(0, q) = 1;
        for (int j = 1; j <= std::min(q, jmax); ++j) {
            const std::int64_t a = at(j - 1, q - 1), b = (j <= q - 1) ? at(j, q - 1) : 0;
            at(j, q) = (a >= kSaturated || b >= kSaturated || a + b >= kSaturated) ? kSaturated
                                                                                  : a + b;
        }
    }
    return t;
}

// sector totals of a box in the reference's mixed-radix order, species 0 most significant
// (markovkit/rdme/population_space.hpp:166-189)
inline std::vector<std::vector<int>> box_totals(const std::vector<int> &limits) {
    const int S = static_cast<int>(limits.size());
    std::vector<std::vector<int>> totals;
    std::vector<int> t(S, 0);
    while (true) {
        totals.push_back(t);
        int s = S - 1;
        while (s >= 0 && t[s] == limits[s]) {
            t[s] = 0;
            --s;
        }
        if (s < 0) {
            break;
        }
        ++t[s];
    }
    return totals;
}

// sectors with the given totals on V voxels, numbered contiguously in list order
inline std::vector<SectorDesc> layout_sectors(int V, int S,
                                              const std::vector<std::vector<int>> &totals,
                                              const BinomTable &bt, std::int64_t *total_size) {
    std::vector<SectorDesc> out;
    std::int64_t begin = 0;
    for (const auto &t : totals) {
        SectorDesc sec;
        std::int64_t comp[kMaxSpecies] = {};
        std::int64_t size = 1;
        int mol = 0;
        for (int s = 0; s < S; ++s) {
            sec.total[s] = t[s];
            sec.mol_offset[s] = mol;
            mol += t[s];
            comp[s] = binom(bt, t[s] + V - 1, t[s]);
            if (comp[s] >= kSaturated || size > std::numeric_limits<std::int64_t>::max() / comp[s]) {
                throw Error(kEOverflow, "population state space is too large");
            }
            size *= comp[s];
        }
        sec.n_mol = mol;
        std::int64_t stride = 1;
        for (int s = S - 1; s >= 0; --s) {
            sec.stride[s] = stride;
            sec.inv_stride[s] = 1.0 / static_cast<double>(stride);
            stride *= comp[s];
        }
        sec.begin = begin;
        sec.size = size;
        for (int r = 0; r < kMaxReactions; ++r) {
            sec.src[r] = -1;
            sec.dst[r] = -1;
        }
        if (begin > std::numeric_limits<std::int64_t>::max() - size) {
            throw Error(kEOverflow, "population state space is too large");
        }
        begin += size;
        out.push_back(sec);
    }
    *total_size = begin;
    return out;
}

// An RDME model: a symmetric voxel graph, volumes, diffusivities and local reactions whose
// rates are tabulated over count tuples 0..tmax_s (markovkit/rdme/reaction_diffusion.hpp).
struct Model {
    int V = 0, S = 0;
    std::vector<int> nbr_ptr, nbr_idx;
    std::vector<double> nbr_w, volumes, diff;
    bool has_grid = false;
    int dim = 0;
    std::int64_t dims[3] = {1, 1, 1};
    double spacing[3] = {1.0, 1.0, 1.0};
    int R = 0;
    std::vector<int> change;   // R x S
    std::vector<int> tmax;     // S
    int nvc = 1;
    std::vector<int> vclass;   // V (empty: one class)
    std::vector<double> rates; // R x nvc x ntuple

    [[nodiscard]] int ntuple() const {
        int n = 1;
        for (int t : tmax) {
            n *= (t + 1);
        }
        return n;
    }

    // grid<D>(dims, spacing): axis 0 fastest, closed boundary, neighbours axis by axis with
    // the lower one first, edge weight = face area / h, volume = product of spacings
    // (conventions pinned by tests/test_rdme.cpp:22-33 of the reference)
    static std::unique_ptr<Model> grid(int dim, const std::int64_t *dims, const double *spacing,
                                       const std::vector<double> &diff) {
        if (dim < 1 || dim > 3) {
            throw Error(kEInval, "grid dimension must be 1, 2 or 3");
        }
        auto m = std::make_unique<Model>();
        m->has_grid = true;
        m->dim = dim;
        std::int64_t V = 1, stride[3] = {1, 1, 1};
        for (int a = 0; a < dim; ++a) {
            if (dims[a] < 1 || !(spacing[a] > 0.0)) {
                throw Error(kEInval, "grid dimensions and spacings must be positive");
            }
            m->dims[a] = dims[a];
            m->spacing[a] = spacing[a];
            stride[a] = V;
            V *= dims[a];
            if (V > (std::int64_t(1) << 30)) {
                throw Error(kEInval, "too many voxels");
            }
        }
        m->V = static_cast<int>(V);
        m->S = static_cast<int>(diff.size());
        m->diff = diff;
        double volume = 1.0;
        for (int a = 0; a < dim; ++a) {
            volume *= spacing[a];
        }
        m->volumes.assign(m->V, volume);
        m->nbr_ptr.assign(m->V + 1, 0);
        for (std::int64_t v = 0; v < V; ++v) {
            std::int64_t rem = v;
            std::int64_t c[3] = {0, 0, 0};
            for (int a = 0; a < dim; ++a) {
                c[a] = rem % dims[a];
                rem /= dims[a];
            }
            for (int a = 0; a < dim; ++a) {
                double face = 1.0;
                for (int b = 0; b < dim; ++b) {
                    if (b != a) {
                        face *= spacing[b];
                    }
                }
                const double w = face / spacing[a];
                if (c[a] > 0) {
                    m->nbr_idx.push_back(static_cast<int>(v - stride[a]));
                    m->nbr_w.push_back(w);
                }
                if (c[a] + 1 < dims[a]) {
                    m->nbr_idx.push_back(static_cast<int>(v + stride[a]));
                    m->nbr_w.push_back(w);
                }
            }
            m->nbr_ptr[v + 1] = static_cast<int>(m->nbr_idx.size());
        }
        return m;
    }

    void validate() const {
        if (V < 1 || S < 1 || S > kMaxSpecies) {
            throw Error(kEInval, "model needs 1..4 species and a voxel");
        }
        if (static_cast<int>(nbr_ptr.size()) != V + 1 || static_cast<int>(volumes.size()) != V ||
            static_cast<int>(diff.size()) != S) {
            throw Error(kEInval, "model arrays have the wrong sizes");
        }
        for (double v : volumes) {
            if (!(v > 0.0) || !std::isfinite(v)) {
                throw Error(kEInval, "voxel_domain: volumes must be positive");
            }
        }
        if (R > kMaxReactions) {
            throw Error(kEInval, "at most 16 local reactions are supported");
        }
        if (R > 0) {
            if (static_cast<int>(change.size()) != R * S || static_cast<int>(tmax.size()) != S ||
                static_cast<std::int64_t>(rates.size()) !=
                    static_cast<std::int64_t>(R) * nvc * ntuple()) {
                throw Error(kEInval, "reaction tables have the wrong sizes");
            }
            if (nvc > 1 && static_cast<int>(vclass.size()) != V) {
                throw Error(kEInval, "one volume class per voxel");
            }
        }
    }
};

// host tables of one voxel graph and model in one precision, and a view over them
template <typename T>
struct HostTables {
    std::vector<int> nbr_ptr, nbr_idx, vclass;
    std::vector<T> in_coef, deg_coef, rate;
    std::vector<unsigned char> vparity;
    std::vector<unsigned> vmask; // structured grids only
    ModelView<T> view; // scalars and masks; pointers set by bind()

    void build(const Model &m, double diff_scale, bool with_reactions, bool absorbing) {
        m.validate();
        const int V = m.V;
        nbr_ptr = m.nbr_ptr;
        nbr_idx = m.nbr_idx;
        const std::size_t E = nbr_idx.size();
        in_coef.assign(E, T(0));
        deg_coef.assign(V, T(0));
        for (int v = 0; v < V; ++v) {
            double deg = 0.0;
            for (int e = m.nbr_ptr[v]; e < m.nbr_ptr[v + 1]; ++e) {
                const int w = m.nbr_idx[e];
                if (w < 0 || w >= V) {
                    throw Error(kEInval, "voxel graph edge out of range");
                }
                deg += m.nbr_w[e] / m.volumes[v];
                // the reverse edge w -> v carries the in-jump
                double wr = -1.0;
                for (int f = m.nbr_ptr[w]; f < m.nbr_ptr[w + 1]; ++f) {
                    if (m.nbr_idx[f] == v) {
                        wr = m.nbr_w[f];
                        break;
                    }
                }
                if (wr < 0.0) {
                    throw Error(kEInval, "voxel graph must list every edge in both directions");
                }
                in_coef[e] = static_cast<T>(wr / m.volumes[w]);
            }
            deg_coef[v] = static_cast<T>(deg);
        }
        vparity.assign(V, 0);
        if (m.has_grid) {
            for (int v = 0; v < V; ++v) {
                std::int64_t rem = v, sum = 0;
                for (int a = 0; a < m.dim; ++a) {
                    sum += rem % m.dims[a];
                    rem /= m.dims[a];
                }
                vparity[v] = static_cast<unsigned char>(sum & 1);
            }
        }
        ModelView<T> mv;
        mv.V = V;
        mv.S = m.S;
        mv.absorbing = absorbing ? 1 : 0;
        for (int s = 0; s < m.S; ++s) {
            mv.diff[s] = static_cast<T>(m.diff[s] * diff_scale);
        }
        vclass.clear();
        rate.clear();
        if (with_reactions && m.R > 0) {
            mv.R = m.R;
            mv.nvc = m.nvc;
            mv.ntuple = m.ntuple();
            int stride = 1;
            for (int s = m.S - 1; s >= 0; --s) {
                mv.tmax[s] = m.tmax[s];
                mv.tstride[s] = stride;
                stride *= m.tmax[s] + 1;
            }
            rate.resize(m.rates.size());
            for (std::size_t k = 0; k < m.rates.size(); ++k) {
                const double a = m.rates[k];
                rate[k] = static_cast<T>((a > 0.0 && std::isfinite(a)) ? a : 0.0);
            }
            if (m.nvc > 1) {
                vclass = m.vclass;
            }
            for (int r = 0; r < m.R; ++r) {
                bool nonneg = true, nonpos = true, fits = true;
                int t_neg = 0;
                for (int s = 0; s < m.S; ++s) {
                    const int c = m.change[r * m.S + s];
                    nonneg = nonneg && c >= 0;
                    nonpos = nonpos && c <= 0;
                    fits = fits && -c <= m.tmax[s];
                    t_neg += (c < 0 ? -c : 0) * mv.tstride[s];
                    mv.change[r][s] = c;
                }
                auto rate_at = [&](int vc, int tuple) {
                    return m.rates[(static_cast<std::size_t>(r) * m.nvc + vc) * mv.ntuple + tuple];
                };
                if (nonneg) {
                    mv.nonneg_mask |= 1U << r;
                    double total = 0.0;
                    for (int v = 0; v < V; ++v) {
                        const double a = rate_at(m.nvc > 1 ? m.vclass[v] : 0, 0);
                        total += (a > 0.0 && std::isfinite(a)) ? a : 0.0;
                    }
                    mv.empty_total[r] = static_cast<T>(total);
                }
                if (nonpos && fits) {
                    for (int vc = 0; vc < m.nvc; ++vc) {
                        if (rate_at(vc, t_neg) > 0.0) {
                            mv.heavy_mask |= 1U << r;
                        }
                    }
                }
            }
        }
        // structured grid with one cell volume: the kernels find neighbours by arithmetic
        bool uniform = m.has_grid && V < (1 << 24);
        for (int v = 0; uniform && v < V; ++v) {
            uniform = m.volumes[v] == m.volumes[0];
        }
        if (uniform) {
            mv.grid_dim = m.dim;
            int stride = 1;
            for (int a = 0; a < 3; ++a) {
                mv.gdims[a] = a < m.dim ? static_cast<int>(m.dims[a]) : 1;
                mv.gstride[a] = stride;
                mv.ginv[a] = 1.0f / static_cast<float>(mv.gdims[a]);
                stride *= mv.gdims[a];
                double face = 1.0;
                for (int b = 0; b < m.dim; ++b) {
                    if (b != a) {
                        face *= m.spacing[b];
                    }
                }
                mv.axis_coef[a] =
                    a < m.dim ? static_cast<T>((face / m.spacing[a]) / m.volumes[0]) : T(0);
            }
            // diffusion only (the multigrid level operators): rows of one molecule per species
            // take the stencil path of visit_row
            mv.stencil = mv.R == 0 ? 1 : 0;
            vmask.assign(V, 0U);
            for (int v = 0; v < V; ++v) {
                std::int64_t rem = v;
                unsigned mask = static_cast<unsigned>(vparity[v]) << kVoxelColourBit;
                for (int a = 0; a < m.dim; ++a) {
                    const std::int64_t c = rem % m.dims[a];
                    rem /= m.dims[a];
                    mask |= (c > 0 ? 1U : 0U) << (2 * a);
                    mask |= (c + 1 < m.dims[a] ? 1U : 0U) << (2 * a + 1);
                }
                vmask[v] = mask;
            }
        } else {
            vmask.clear();
        }
        view = mv;
        bind_host();
    }

    // point the view at the host vectors
    void bind_host() {
        view.nbr_ptr = nbr_ptr.data();
        view.nbr_idx = nbr_idx.data();
        view.in_coef = in_coef.data();
        view.deg_coef = deg_coef.data();
        view.vparity = vparity.data();
        view.vmask = vmask.empty() ? nullptr : vmask.data();
        view.vclass = vclass.empty() ? nullptr : vclass.data();
        view.rate = rate.empty() ? nullptr : rate.data();
    }
};

// reaction couplings between the sectors of one level (src/dst/heavy), as the reference's
// generator finds them with space.find (markovkit/generator.hpp:30-37)
template <typename T>
void couple_sectors(std::vector<SectorDesc> &sectors, int S, const Model &m,
                    const ModelView<T> &mv, bool with_reactions) {
    std::map<std::vector<int>, int> by_totals;
    for (std::size_t k = 0; k < sectors.size(); ++k) {
        by_totals[std::vector<int>(sectors[k].total, sectors[k].total + S)] = static_cast<int>(k);
    }
    for (auto &sec : sectors) {
        sec.heavy = 0;
        for (int r = 0; r < kMaxReactions; ++r) {
            sec.src[r] = -1;
            sec.dst[r] = -1;
        }
        if (!with_reactions) {
            continue;
        }
        for (int r = 0; r < m.R; ++r) {
            std::vector<int> up(S), down(S);
            for (int s = 0; s < S; ++s) {
                up[s] = sec.total[s] + m.change[r * S + s];
                down[s] = sec.total[s] - m.change[r * S + s];
            }
            auto it = by_totals.find(up);
            sec.dst[r] = it == by_totals.end() ? -1 : it->second;
            it = by_totals.find(down);
            sec.src[r] = it == by_totals.end() ? -1 : it->second;
            if (((mv.heavy_mask >> r) & 1U) && sec.src[r] >= 0) {
                sec.heavy = 1;
            }
        }
    }
}

// coarsen (markovkit/rdme/multigrid.hpp:23-42): halve every axis longer than one cell and
// double its spacing; false when an axis is odd or no axis is long
inline bool coarsen_grid(int dim, const std::int64_t *dims, const double *spacing,
                         std::int64_t *cdims, double *cspacing) {
    bool reduced = false;
    for (int a = 0; a < 3; ++a) {
        cdims[a] = dims[a];
        cspacing[a] = spacing[a];
    }
    for (int a = 0; a < dim; ++a) {
        if (dims[a] == 1) {
            continue;
        }
        if (dims[a] % 2 != 0) {
            return false;
        }
        cdims[a] = dims[a] / 2;
        cspacing[a] = spacing[a] * 2.0;
        reduced = true;
    }
    return reduced;
}

// the coarse voxel containing each fine voxel, and log(children) of each coarse voxel
// (markovkit/rdme/multigrid.hpp:54-65)
inline void parent_map(int dim, const std::int64_t *dims, const std::int64_t *cdims,
                       std::vector<int> &parent, std::vector<double> &log_children) {
    std::int64_t Vf = 1, Vc = 1;
    for (int a = 0; a < dim; ++a) {
        Vf *= dims[a];
        Vc *= cdims[a];
    }
    parent.assign(static_cast<std::size_t>(Vf), 0);
    std::vector<int> children(static_cast<std::size_t>(Vc), 0);
    for (std::int64_t v = 0; v < Vf; ++v) {
        std::int64_t rem = v, cv = 0, cstride = 1;
        for (int a = 0; a < dim; ++a) {
            std::int64_t c = rem % dims[a];
            rem /= dims[a];
            if (dims[a] > 1) {
                c /= 2;
            }
            cv += c * cstride;
            cstride *= cdims[a];
        }
        parent[v] = static_cast<int>(cv);
        ++children[cv];
    }
    log_children.resize(static_cast<std::size_t>(Vc));
    for (std::int64_t a = 0; a < Vc; ++a) {
        log_children[a] = std::log(static_cast<double>(children[a]));
    }
}

// the largest total of one species in any sector (sizes the kernels' molecule lists)
inline int max_species_total(const std::vector<SectorDesc> &sectors) {
    int m = 0;
    for (const auto &s : sectors) {
        for (int k = 0; k < kMaxSpecies; ++k) {
            m = std::max(m, s.total[k]);
        }
    }
    return m;
}

} // namespace mkb
