// Test infrastructure: runs the product's shared host/device row logic
// (markovkit_b200/csrc/generator_row.cuh, population_index.cuh, host_model.hpp) on the CPU,
// one row at a time, so the non-GPU tests can check state indexing, the generator gather and
// the multigrid transfer against the reference's golden vectors before any kernel runs.
// Built by tests/cpu_emulator.py with g++ into a small shared library.
#include "host_model.hpp"
#include "pair_rows.cuh"
#include "stencil_row.cuh"

#include <cstdint>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

using namespace mkb;

namespace {

struct Problem {
    std::unique_ptr<Model> model;
    std::vector<std::int64_t> binom;
    BinomTable B;
    std::vector<SectorDesc> sectors;
    std::int64_t n = 0;
    HostTables<double> t;
};

void write_err(char *err, const std::string &msg) {
    if (err) {
        std::strncpy(err, msg.c_str(), 255);
        err[255] = '\0';
    }
}

Problem make(int dim, const std::int64_t *dims, const double *spacing, int S, const double *D,
             int R, const int *change, const int *tmax, const double *rates, int is_box,
             const int *limits, int absorbing, int csr = 0) {
    Problem p;
    p.model = Model::grid(dim, dims, spacing, std::vector<double>(D, D + S));
    if (R > 0) {
        p.model->R = R;
        p.model->change.assign(change, change + R * S);
        p.model->tmax.assign(tmax, tmax + S);
        p.model->rates.assign(rates, rates + static_cast<std::size_t>(R) * p.model->ntuple());
    }
    const std::vector<int> lim(limits, limits + S);
    const int max_total = *std::max_element(lim.begin(), lim.end());
    p.binom = binomial_table(max_total + 1, p.model->V + max_total + 1);
    p.B = {p.binom.data(), max_total + 1, p.model->V + max_total + 1};
    const auto totals = is_box ? box_totals(lim) : std::vector<std::vector<int>>{lim};
    p.sectors = layout_sectors(p.model->V, S, totals, p.B, &p.n);
    if (csr == 1) {
        // the same voxel graph given as explicit neighbour lists (the general-graph path)
        p.model->has_grid = false;
    }
    p.t.build(*p.model, 1.0, true, absorbing != 0);
    if (csr == 2) {
        // the structured grid through the general row visit (no stencil path)
        p.t.view.stencil = 0;
    }
    couple_sectors<double>(p.sectors, S, *p.model, p.t.view, true);
    return p;
}

constexpr int kCap = 64;
using State = RowState<kMaxSpecies, kCap>; // the generic shape: any species count up to 4

// the shapes the stencil kernel serves (stencil_shape in row_kernels.cu)
bool stencil_shape_host(int S, int cap) { return (S == 1 && cap <= 4) || (S == 2 && cap <= 1); }

} // namespace

extern "C" {

// exit, leak, Q x and (shift I - Q) x for every state; returns the number of states
std::int64_t emu_generator(int dim, const std::int64_t *dims, const double *spacing, int S,
                           const double *D, int R, const int *change, const int *tmax,
                           const double *rates, int is_box, const int *limits, int absorbing,
                           double shift, const double *x, double *exit_out, double *leak_out,
                           double *Qx, double *Ax, char *err, int csr) {
    try {
        Problem p =
            make(dim, dims, spacing, S, D, R, change, tmax, rates, is_box, limits, absorbing, csr);
        if (!x) {
            return p.n;
        }
        // the state shape the device kernels use for this space
        with_shape(S, max_species_total(p.sectors), [&]<int NS, int TMAX>() {
            for (const SectorDesc &sec : p.sectors) {
                for (std::int64_t local = 0; local < sec.size; ++local) {
                    RowState<NS, TMAX> st;
                    load_state<NS, TMAX>(p.B, sec, S, p.model->V, local, st);
                    double e = 0.0, l = 0.0, in = 0.0;
                    visit_row<double, NS, TMAX>(
                        p.B, p.sectors.data(), sec, p.t.view, local, st, true, 0, 1, e, l,
                        [&](std::int64_t j, double a, double) {
                            if (j < 0 || j >= p.n) {
                                throw Error(kEInval, "in-jump source out of range");
                            }
                            in += a * x[j];
                        });
                    const std::int64_t i = sec.begin + local;
                    exit_out[i] = e;
                    leak_out[i] = l;
                    Qx[i] = in - e * x[i];
                    Ax[i] = (shift + e) * x[i] - in;
                }
            }
            return 0;
        });
        return p.n;
    } catch (const std::exception &e) {
        write_err(err, e.what());
        return -1;
    }
}

// The stencil row forms (stencil_row.cuh) against the general row visit on every light row of
// a stencil-shaped space: the same in-jumps (source and rate, bit for bit) in the same order, the
// same exit and leak bits, the same colour. Returns the rows compared (-1 with err on the first
// difference; 0 when the space has no stencil shape).
std::int64_t emu_stencil_check(int dim, const std::int64_t *dims, const double *spacing, int S,
                               const double *D, int R, const int *change, const int *tmax,
                               const double *rates, int is_box, const int *limits, int absorbing,
                               char *err) {
    try {
        Problem p = make(dim, dims, spacing, S, D, R, change, tmax, rates, is_box, limits, absorbing);
        const int cap = max_species_total(p.sectors);
        if (!stencil_shape_host(S, cap) || !p.t.view.vmask) {
            return 0;
        }
        std::int64_t rows = 0;
        // the pair and single-molecule forms: the same in-jumps (as a multiset: reactions may
        // come in another order) and the same exit and leak to rounding
        std::vector<StencilSector<double>> tabs;
        std::vector<double> ddeg;
        StencilView<double> sv;
        if (build_stencil_tables<double>(p.sectors, S, cap, p.t.view, p.t.rate, p.t.deg_coef, tabs,
                                         ddeg, sv)) {
            sv.sectors = tabs.data();
            sv.ddeg = ddeg.data();
            with_shape(S, cap, [&]<int NS, int TMAX>() {
                for (std::size_t k = 0; k < p.sectors.size(); ++k) {
                    const SectorDesc &sec = p.sectors[k];
                    const StencilSector<double> &ss = tabs[k];
                    if (sec.heavy && S == 1 && ss.fast && ss.heavy_ok) {
                        // rows with in-jumps from every voxel: the pair-form heavy terms
                        for (std::int64_t local = 0; local < sec.size; ++local) {
                            RowState<NS, TMAX> st;
                            load_state<NS, TMAX>(p.B, sec, S, p.model->V, local, st);
                            std::vector<std::pair<std::int64_t, double>> a, b;
                            double e1 = 0, l1 = 0;
                            visit_row<double, NS, TMAX>(p.B, p.sectors.data(), sec, p.t.view, local, st,
                                                        false, 0, 1, e1, l1,
                                                        [&](std::int64_t j, double r, double) { a.emplace_back(j, r); });
                            pair_heavy_terms<double>(ss, p.model->V, ss.total[0], static_cast<int>(local), 0, 1,
                                                     [&](int j, double r, bool on) {
                                                         if (on) {
                                                             b.emplace_back(j, r);
                                                         }
                                                     });
                            std::sort(a.begin(), a.end());
                            std::sort(b.begin(), b.end());
                            if (a != b) {
                                throw Error(kEInval, "pair heavy terms differ at row " +
                                                         std::to_string(sec.begin + local) + " (" +
                                                         std::to_string(a.size()) + " vs " +
                                                         std::to_string(b.size()) + ")");
                            }
                            ++rows;
                        }
                        continue;
                    }
                    if (sec.heavy || !ss.fast) {
                        continue;
                    }
                    for (std::int64_t local = 0; local < sec.size; ++local) {
                        RowState<NS, TMAX> st;
                        load_state<NS, TMAX>(p.B, sec, S, p.model->V, local, st);
                        std::vector<std::pair<std::int64_t, double>> a, b;
                        double e1 = 0, l1 = 0, e2 = 0, l2 = 0;
                        visit_row<double, NS, TMAX>(p.B, p.sectors.data(), sec, p.t.view, local, st,
                                                    true, 0, 1, e1, l1,
                                                    [&](std::int64_t j, double r, double) { a.emplace_back(j, r); });
                        const int row = static_cast<int>(sec.begin + local);
                        const int V = p.model->V;
                        int u0 = 0, u1 = 0;
                        unsigned m0 = 0, m1 = 0;
                        auto acc = [&](int j, double r, bool on) {
                            if (on) {
                                b.emplace_back(j, r);
                            }
                        };
                        if (S == 1) {
                            const int t = ss.total[0];
                            if (t == 2) {
                                unrank_pair(static_cast<int>(local), u0, u1);
                                m1 = p.t.vmask[V - 1 - u1];
                            } else {
                                u0 = static_cast<int>(local);
                            }
                            if (t >= 1) {
                                m0 = p.t.vmask[V - 1 - u0];
                            }
                            for (int q = 0; q < t; ++q) {
                                if ((q == 0 ? u0 : u1) != st.u[0][q]) {
                                    throw Error(kEInval, "pair unrank differs at row " + std::to_string(row));
                                }
                            }
                            pair_row<double, true>(p.t.view, sv, ss, t, u0, u1, m0, m1, row, e2, l2, acc);
                        } else {
                            if (ss.total[0] && ss.total[1]) {
                                u0 = static_cast<int>(local) / ss.stride0;
                                u1 = static_cast<int>(local) - u0 * ss.stride0;
                            } else {
                                u0 = u1 = static_cast<int>(local);
                            }
                            if (ss.total[0]) {
                                m0 = p.t.vmask[V - 1 - u0];
                            }
                            if (ss.total[1]) {
                                m1 = p.t.vmask[V - 1 - u1];
                            }
                            singles_row<double, true>(p.t.view, sv, ss, u0, u1, m0, m1, row, e2, l2, acc);
                        }
                        std::sort(a.begin(), a.end());
                        std::sort(b.begin(), b.end());
                        const double tol = 1e-14 * (std::abs(e1) + 1e-300);
                        if (a != b || std::abs(e1 - e2) > tol || std::abs(l1 - l2) > 1e-14 * (std::abs(l1) + 1e-300) + 1e-300 ||
                            ((((m0 ^ m1) >> kVoxelColourBit) & 1U) != static_cast<unsigned>(state_colour<double, NS, TMAX>(p.t.view, sec, st)))) {
                            throw Error(kEInval, "pair row differs at row " + std::to_string(row) + " (" +
                                                     std::to_string(a.size()) + " vs " + std::to_string(b.size()) +
                                                     " in-jumps, exit " + std::to_string(e1) + " vs " + std::to_string(e2) + ")");
                        }
                        ++rows;
                    }
                }
                return 0;
            });
        }
        with_stencil_shape(S, cap, [&]<int NS, int TMAX>() {
            for (const SectorDesc &sec : p.sectors) {
                if (sec.heavy) {
                    continue;
                }
                for (std::int64_t local = 0; local < sec.size; ++local) {
                    RowState<NS, TMAX> st;
                    load_state<NS, TMAX>(p.B, sec, S, p.model->V, local, st);
                    StencilState<NS, TMAX> ss;
                    stencil_load<double, NS, TMAX>(sec, p.t.view, static_cast<int>(local), ss);
                    for (int s2 = 0; s2 < NS; ++s2) {
                        for (int q = 0; q < (s2 < S ? sec.total[s2] : 0); ++q) {
                            if (st.u[s2][q] != ss.rs.u[s2][q]) {
                                throw Error(kEInval, "unrank differs at row " + std::to_string(sec.begin + local));
                            }
                        }
                    }
                    std::vector<std::pair<std::int64_t, double>> a, b;
                    double e1 = 0, l1 = 0, e2 = 0, l2 = 0;
                    visit_row<double, NS, TMAX>(p.B, p.sectors.data(), sec, p.t.view, local, st, true, 0,
                                                1, e1, l1, [&](std::int64_t j, double r, double) { a.emplace_back(j, r); });
                    const int row = static_cast<int>(sec.begin + local);
                    stencil_visit<double, NS, TMAX, true>(p.B, p.sectors.data(), sec, p.t.view, ss, row,
                                                          e2, l2, [&](int j, double r, double) { b.emplace_back(j, r); });
                    if (a != b || e1 != e2 || l1 != l2 ||
                        state_colour<double, NS, TMAX>(p.t.view, sec, st) != stencil_colour<NS, TMAX>(ss)) {
                        throw Error(kEInval, "stencil row differs at row " + std::to_string(row) + " (" +
                                                 std::to_string(a.size()) + " vs " + std::to_string(b.size()) +
                                                 " in-jumps)");
                    }
                    ++rows;
                }
            }
            return 0;
        });
        return rows;
    } catch (const std::exception &e) {
        write_err(err, e.what());
        return -1;
    }
}

// the triplets of sign * (Q - shift I) row by row, as the device assembly makes them: each
// row's diagonal -sign (exit + shift), then sign * rate for each in-jump in visit order.
// Returns the triplet count; writes them when it is at most `capacity`.
std::int64_t emu_matrix(int dim, const std::int64_t *dims, const double *spacing, int S,
                        const double *D, int R, const int *change, const int *tmax,
                        const double *rates, int is_box, const int *limits, int absorbing,
                        double shift, double sign, std::int64_t *row, std::int64_t *col,
                        double *val, std::int64_t capacity, char *err, int csr) {
    try {
        Problem p =
            make(dim, dims, spacing, S, D, R, change, tmax, rates, is_box, limits, absorbing, csr);
        std::int64_t k = 0;
        const auto put = [&](std::int64_t i, std::int64_t j, double v) {
            if (k < capacity) {
                row[k] = i;
                col[k] = j;
                val[k] = v;
            }
            ++k;
        };
        with_shape(S, max_species_total(p.sectors), [&]<int NS, int TMAX>() {
            for (const SectorDesc &sec : p.sectors) {
                for (std::int64_t local = 0; local < sec.size; ++local) {
                    RowState<NS, TMAX> st;
                    load_state<NS, TMAX>(p.B, sec, S, p.model->V, local, st);
                    const std::int64_t i = sec.begin + local;
                    std::vector<std::pair<std::int64_t, double>> in;
                    double e = 0.0, l = 0.0;
                    visit_row<double, NS, TMAX>(p.B, p.sectors.data(), sec, p.t.view, local, st,
                                                true, 0, 1, e, l,
                                                [&](std::int64_t j, double a, double) {
                                                    if (j < 0 || j >= p.n) {
                                                        throw Error(kEInval, "in-jump source out of range");
                                                    }
                                                    in.emplace_back(j, a);
                                                });
                    put(i, i, -sign * (e + shift));
                    for (const auto &[j, a] : in) {
                        put(i, j, sign * a);
                    }
                }
            }
            return 0;
        });
        return k;
    } catch (const std::exception &e) {
        write_err(err, e.what());
        return -1;
    }
}

// states (n x V*S, voxel-major) of every index by the product's unrank, and the product's
// rank of each of them
std::int64_t emu_states(int V, int S, const int *limits, int is_box, int *states,
                        std::int64_t *ranks, char *err) {
    try {
        const std::vector<int> lim(limits, limits + S);
        const int max_total = *std::max_element(lim.begin(), lim.end());
        auto table = binomial_table(max_total + 1, V + max_total + 1);
        const BinomTable B{table.data(), max_total + 1, V + max_total + 1};
        const auto totals = is_box ? box_totals(lim) : std::vector<std::vector<int>>{lim};
        std::int64_t n = 0;
        const auto sectors = layout_sectors(V, S, totals, B, &n);
        if (!states) {
            return n;
        }
        for (const SectorDesc &sec : sectors) {
            for (std::int64_t local = 0; local < sec.size; ++local) {
                State st;
                load_state<kMaxSpecies, kCap>(B, sec, S, V, local, st);
                int *out = states + (sec.begin + local) * static_cast<std::int64_t>(V) * S;
                std::fill(out, out + static_cast<std::int64_t>(V) * S, 0);
                std::int64_t r = sec.begin;
                for (int s = 0; s < S; ++s) {
                    for (int q = 0; q < sec.total[s]; ++q) {
                        ++out[static_cast<std::int64_t>(V - 1 - st.u[s][q]) * S + s];
                    }
                    r += rank_species<kCap>(B, st.u[s], sec.total[s]) * sec.stride[s];
                }
                ranks[sec.begin + local] = r;
            }
        }
        return n;
    } catch (const std::exception &e) {
        write_err(err, e.what());
        return -1;
    }
}

// population_transfer of one sector between a grid and its coarsening:
// Pc = prolong(c), Rg = restrict(g); returns the fine size (coarse size in *n_coarse)
std::int64_t emu_transfer(int dim, const std::int64_t *dims, const double *spacing, int S,
                          const int *totals, const double *c, const double *g, double *Pc,
                          double *Rg, std::int64_t *n_coarse, char *err) {
    try {
        std::int64_t cdims[3];
        double cspacing[3];
        if (!coarsen_grid(dim, dims, spacing, cdims, cspacing)) {
            throw Error(kEInval, "grid cannot be coarsened");
        }
        std::int64_t Vf = 1, Vc = 1;
        for (int a = 0; a < dim; ++a) {
            Vf *= dims[a];
            Vc *= cdims[a];
        }
        const std::vector<int> t(totals, totals + S);
        const int max_total = *std::max_element(t.begin(), t.end());
        auto table = binomial_table(max_total + 1, static_cast<int>(Vf) + max_total + 1);
        const BinomTable B{table.data(), max_total + 1, static_cast<int>(Vf) + max_total + 1};
        std::int64_t nf = 0, nc = 0;
        auto fine = layout_sectors(static_cast<int>(Vf), S, {t}, B, &nf);
        auto coarse = layout_sectors(static_cast<int>(Vc), S, {t}, B, &nc);
        fine[0].coarse = 0;
        *n_coarse = nc;
        if (!c) {
            return nf;
        }
        std::vector<int> parent;
        std::vector<double> log_children, lgf(max_total + 2);
        parent_map(dim, dims, cdims, parent, log_children);
        for (std::size_t k = 0; k < lgf.size(); ++k) {
            lgf[k] = std::lgamma(static_cast<double>(k) + 1.0);
        }
        TransferView tv;
        tv.Vc = static_cast<int>(Vc);
        tv.parent = parent.data();
        tv.log_children = log_children.data();
        tv.lgf = lgf.data();
        tv.coarse_sectors = coarse.data();
        std::fill(Rg, Rg + nc, 0.0);
        with_shape(S, max_total, [&]<int NS, int TMAX>() {
            for (std::int64_t i = 0; i < nf; ++i) {
                RowState<NS, TMAX> st;
                load_state<NS, TMAX>(B, fine[0], S, static_cast<int>(Vf), i, st);
                double w = 0.0;
                const std::int64_t ci =
                    coarse_index<NS, TMAX>(B, tv, fine[0], static_cast<int>(Vf), st, &w);
                if (ci < 0 || ci >= nc) {
                    throw Error(kEInval, "coarse index out of range");
                }
                Pc[i] = w * c[ci];
                Rg[ci] += g[i];
            }
            return 0;
        });
        return nf;
    } catch (const std::exception &e) {
        write_err(err, e.what());
        return -1;
    }
}

} // extern "C"
