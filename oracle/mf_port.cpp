// ORACLE TEST INFRASTRUCTURE — matrix-free CPU restatement ("port") of MarkovKit's RDME
// resolvent path, for sizes where the reference's own containers do not fit in memory and as
// the bounded CPU baseline. Not part of the product, and written independently of it.
//
// It restates, with OpenMP over rows:
//  * population_box numbering (markovkit/rdme/population_space.hpp:32-100,131-189): sectors in
//    mixed-radix order of their totals, states of a sector lexicographic with species 0 most
//    significant and voxel 0's count most significant. A species' composition is ranked as the
//    combination-with-repetition of its molecules: with u = V-1-voxel sorted ascending,
//    rank = sum_p C(u_p + p, p + 1) (stars and bars; equal to the reference's rank);
//  * the generator of reaction_diffusion (reaction_diffusion.hpp:82-118, generator.hpp:27-81),
//    applied as a gather over rows;
//  * sector_multigrid (multigrid.hpp:25-228,309-317,369-403): per sector, a geometric hierarchy
//    with doubled diffusivity per level, multinomial prolongation, aggregation restriction,
//    weighted Jacobi 2/2 sweeps, a dense LU at the bottom;
//  * restarted GMRES with right preconditioning and modified Gram-Schmidt (Saad, Alg. 9.5), as
//    the numerics shim states it.
//
// usage: mf_port key=value ...  (dim cells h cap model birth death k D D2 shift rhs seed tol
//        restart maxit solves warmup threads sample_iters out)
#include "seeded.hpp"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using i64 = std::int64_t;
using vec = std::vector<double>;

// ---- grid ----------------------------------------------------------------------------------
struct Grid {
    int dim = 1;
    i64 dims[3] = {1, 1, 1};
    double h[3] = {1, 1, 1};
    int V = 1;
    std::vector<std::vector<std::pair<int, double>>> nbr; // (to, weight)
    double volume = 1;

    Grid(int d, const i64 *n, const double *sp) : dim(d) {
        i64 stride[3] = {1, 1, 1};
        i64 total = 1;
        for (int a = 0; a < d; ++a) {
            dims[a] = n[a];
            h[a] = sp[a];
            stride[a] = total;
            total *= n[a];
        }
        V = static_cast<int>(total);
        volume = 1;
        for (int a = 0; a < d; ++a) {
            volume *= h[a];
        }
        nbr.resize(V);
        for (int v = 0; v < V; ++v) {
            i64 rem = v, c[3] = {0, 0, 0};
            for (int a = 0; a < d; ++a) {
                c[a] = rem % dims[a];
                rem /= dims[a];
            }
            for (int a = 0; a < d; ++a) {
                double face = 1;
                for (int b = 0; b < d; ++b) {
                    if (b != a) {
                        face *= h[b];
                    }
                }
                if (c[a] > 0) {
                    nbr[v].push_back({static_cast<int>(v - stride[a]), face / h[a]});
                }
                if (c[a] + 1 < dims[a]) {
                    nbr[v].push_back({static_cast<int>(v + stride[a]), face / h[a]});
                }
            }
        }
    }
};

// ---- combinatorics -------------------------------------------------------------------------
struct Choose {
    std::vector<std::vector<i64>> c; // c[j][q] = C(q, j)
    Choose(int jmax, int qmax) : c(jmax + 1, std::vector<i64>(qmax + 1, 0)) {
        for (int q = 0; q <= qmax; ++q) {
            c[0][q] = 1;
        }
        for (int j = 1; j <= jmax; ++j) {
            for (int q = j; q <= qmax; ++q) {
                c[j][q] = c[j - 1][q - 1] + c[j][q - 1];
            }
        }
    }
    i64 operator()(int q, int j) const { return (q < 0 || q < j) ? 0 : c[j][q]; }
};

// a sector: fixed totals; its states are mixed-radix products of per-species compositions
struct Sector {
    std::vector<int> totals;
    std::vector<i64> comp, weight; // per species: number of compositions, mixed-radix weight
    i64 begin = 0, size = 0;
};

struct Space {
    int V = 0, S = 0;
    const Choose *C = nullptr;
    std::vector<Sector> sectors;
    std::map<std::vector<int>, int> index;
    i64 n = 0;

    void add(const std::vector<int> &t) {
        Sector s;
        s.totals = t;
        s.size = 1;
        for (int k = 0; k < S; ++k) {
            s.comp.push_back((*C)(t[k] + V - 1, t[k]));
            s.size *= s.comp.back();
        }
        s.weight.assign(S, 1);
        for (int k = S - 2; k >= 0; --k) {
            s.weight[k] = s.weight[k + 1] * s.comp[k + 1];
        }
        s.begin = n;
        n += s.size;
        index[t] = static_cast<int>(sectors.size());
        sectors.push_back(s);
    }
    int sector_of(i64 i) const {
        int lo = 0, hi = static_cast<int>(sectors.size()) - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (sectors[mid].begin <= i) {
                lo = mid;
            } else {
                hi = mid - 1;
            }
        }
        return lo;
    }
    // molecules (voxels, one list per species) of state i
    void state(i64 i, int &k, std::vector<std::vector<int>> &mol) const {
        k = sector_of(i);
        const Sector &s = sectors[k];
        i64 rem = i - s.begin;
        mol.assign(S, {});
        for (int sp = 0; sp < S; ++sp) {
            i64 r = rem / s.weight[sp];
            rem -= r * s.weight[sp];
            const int t = s.totals[sp];
            std::vector<int> u(t);
            int hi = V - 1 + t - 1;
            for (int j = t; j >= 1; --j) {
                int q = j - 1;
                int lo = j - 1, up = hi;
                while (lo < up) {
                    const int mid = (lo + up + 1) / 2;
                    if ((*C)(mid, j) <= r) {
                        lo = mid;
                    } else {
                        up = mid - 1;
                    }
                }
                q = lo;
                u[j - 1] = q - (j - 1);
                r -= (*C)(q, j);
                hi = q - 1;
            }
            for (int p = 0; p < t; ++p) {
                mol[sp].push_back(V - 1 - u[p]);
            }
        }
    }
    // index of a state given by molecule voxels (any order), -1 if its totals are absent
    i64 find(const std::vector<std::vector<int>> &mol) const {
        std::vector<int> t(S);
        for (int sp = 0; sp < S; ++sp) {
            t[sp] = static_cast<int>(mol[sp].size());
        }
        auto it = index.find(t);
        if (it == index.end()) {
            return -1;
        }
        const Sector &s = sectors[it->second];
        i64 r = s.begin;
        for (int sp = 0; sp < S; ++sp) {
            std::vector<int> u;
            for (int v : mol[sp]) {
                u.push_back(V - 1 - v);
            }
            std::sort(u.begin(), u.end());
            i64 rs = 0;
            for (int p = 0; p < static_cast<int>(u.size()); ++p) {
                rs += (*C)(u[p] + p, p + 1);
            }
            r += rs * s.weight[sp];
        }
        return r;
    }
};

// ---- model ---------------------------------------------------------------------------------
struct Reaction {
    std::vector<int> change;
    std::function<double(const std::vector<int> &, double)> rate;
};

// one level operator: A = shift I - Q on a space over a grid, rows assembled once as a gather
// list (the port keeps rows explicitly; the sizes it serves fit in host memory)
struct Operator {
    i64 n = 0;
    std::vector<i64> ptr;
    std::vector<i64> col;
    std::vector<double> val; // off-diagonal in-rates (positive)
    vec exit;

    void build(const Space &sp, const Grid &g, const std::vector<double> &D,
               const std::vector<Reaction> &rx, bool absorbing) {
        n = sp.n;
        exit.assign(n, 0.0);
        // out-jumps scattered into per-target lists, then packed by target row (gather form)
        std::vector<std::vector<std::pair<i64, double>>> in(n);
        const int nt = omp_get_max_threads();
        std::vector<std::vector<std::pair<i64, std::pair<i64, double>>>> local(nt);
#pragma omp parallel
        {
            auto &out = local[omp_get_thread_num()];
            std::vector<std::vector<int>> mol;
#pragma omp for schedule(dynamic, 4096)
            for (i64 j = 0; j < n; ++j) {
                int k;
                sp.state(j, k, mol);
                double ex = 0.0;
                // counts per voxel
                std::map<int, std::vector<int>> counts;
                for (int s = 0; s < sp.S; ++s) {
                    for (int v : mol[s]) {
                        counts[v].resize(sp.S, 0);
                        counts[v][s] += 1;
                    }
                }
                // diffusion (reaction_diffusion.hpp:85-98)
                for (auto &[v, c] : counts) {
                    for (auto [w, weight] : g.nbr[v]) {
                        for (int s = 0; s < sp.S; ++s) {
                            if (c[s] == 0) {
                                continue;
                            }
                            auto m2 = mol;
                            auto pos = std::find(m2[s].begin(), m2[s].end(), v);
                            *pos = w;
                            const double rate = c[s] * D[s] * weight / g.volume;
                            out.push_back({sp.find(m2), {j, rate}});
                            ex += rate;
                        }
                    }
                }
                // local reactions in every voxel (reaction_diffusion.hpp:99-116). An empty voxel
                // whose reaction lands outside the space only adds to the exit rate, so those
                // voxels are counted instead of visited.
                std::vector<int> tot(sp.S, 0);
                for (int s = 0; s < sp.S; ++s) {
                    tot[s] = static_cast<int>(mol[s].size());
                }
                std::vector<char> visit_empty(rx.size(), 0);
                const std::vector<int> zero(sp.S, 0);
                const int n_empty = g.V - static_cast<int>(counts.size());
                for (size_t q = 0; q < rx.size(); ++q) {
                    const Reaction &r = rx[q];
                    const double rate = r.rate(zero, g.volume);
                    bool valid = rate > 0.0;
                    std::vector<int> t2 = tot;
                    for (int s = 0; s < sp.S; ++s) {
                        valid = valid && r.change[s] >= 0;
                        t2[s] += r.change[s];
                    }
                    if (!valid) {
                        continue;
                    }
                    if (sp.index.count(t2)) {
                        visit_empty[q] = 1;
                    } else if (absorbing) {
                        ex += rate * n_empty;
                    }
                }
                for (int v = 0; v < g.V; ++v) {
                    auto it = counts.find(v);
                    const bool empty = it == counts.end();
                    std::vector<int> c = empty ? zero : it->second;
                    for (size_t q = 0; q < rx.size(); ++q) {
                        if (empty && !visit_empty[q]) {
                            continue;
                        }
                        const Reaction &r = rx[q];
                        const double rate = r.rate(c, g.volume);
                        if (!(rate > 0.0)) {
                            continue;
                        }
                        bool valid = true;
                        for (int s = 0; s < sp.S; ++s) {
                            valid = valid && c[s] + r.change[s] >= 0;
                        }
                        if (!valid) {
                            continue;
                        }
                        auto m2 = mol;
                        for (int s = 0; s < sp.S; ++s) {
                            for (int q = 0; q < r.change[s]; ++q) {
                                m2[s].push_back(v);
                            }
                            for (int q = 0; q < -r.change[s]; ++q) {
                                m2[s].erase(std::find(m2[s].begin(), m2[s].end(), v));
                            }
                        }
                        const i64 target = sp.find(m2);
                        if (target >= 0) {
                            out.push_back({target, {j, rate}});
                            ex += rate;
                        } else if (absorbing) {
                            ex += rate;
                        }
                    }
                }
                exit[j] = ex;
            }
        }
        for (auto &out : local) {
            for (auto &[row, e] : out) {
                in[row].push_back(e);
            }
            out.clear();
            out.shrink_to_fit();
        }
        ptr.assign(n + 1, 0);
        for (i64 i = 0; i < n; ++i) {
            ptr[i + 1] = ptr[i] + static_cast<i64>(in[i].size());
        }
        col.resize(ptr[n]);
        val.resize(ptr[n]);
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            std::sort(in[i].begin(), in[i].end());
            i64 p = ptr[i];
            for (auto &[c, v] : in[i]) {
                col[p] = c;
                val[p++] = v;
            }
        }
    }

    // y = shift x - Q x
    void apply(double shift, const double *x, double *y) const {
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            double s = (shift + exit[i]) * x[i];
            for (i64 p = ptr[i]; p < ptr[i + 1]; ++p) {
                s -= val[p] * x[col[p]];
            }
            y[i] = s;
        }
    }
};

// ---- population multigrid of one sector ----------------------------------------------------
struct Level {
    Space space;
    Grid grid;
    Operator A;
    std::unique_ptr<Level> coarse;
    std::vector<i64> coarse_of;
    vec weight;
    std::vector<double> lu; // terminal dense LU (row-major) and its pivots
    std::vector<int> piv;
    mutable vec rhs, x, r, e, tmp, crhs, cx;
    Level(const Grid &g) : grid(g) {}
};

struct Options {
    int pre = 2, post = 2;
    double omega = 2.0 / 3.0;
    i64 coarsest = 4;
    int max_levels = 32;
};

std::unique_ptr<Level> build_level(const Grid &g, const std::vector<double> &D,
                                   const std::vector<int> &totals, double shift,
                                   const Options &o, int levels_left, const Choose &C) {
    auto L = std::make_unique<Level>(g);
    L->space.V = g.V;
    L->space.S = static_cast<int>(totals.size());
    L->space.C = &C;
    L->space.add(totals);
    L->A.build(L->space, g, D, {}, true);
    const i64 n = L->space.n;
    L->rhs.assign(n, 0);
    L->x.assign(n, 0);
    L->r.assign(n, 0);
    L->e.assign(n, 0);
    L->tmp.assign(n, 0);
    // coarsen (multigrid.hpp:25-42)
    i64 cd[3] = {g.dims[0], g.dims[1], g.dims[2]};
    double ch[3] = {g.h[0], g.h[1], g.h[2]};
    bool ok = false;
    for (int a = 0; a < g.dim; ++a) {
        if (g.dims[a] == 1) {
            continue;
        }
        if (g.dims[a] % 2) {
            ok = false;
            cd[0] = -1;
            break;
        }
        cd[a] /= 2;
        ch[a] *= 2;
        ok = true;
    }
    if (n <= o.coarsest || levels_left <= 1 || !ok || cd[0] < 0) {
        // dense LU of the whole level (multigrid.hpp:154-158,247-264)
        const int m = static_cast<int>(n);
        L->lu.assign(static_cast<size_t>(m) * m, 0.0);
        for (int i = 0; i < m; ++i) {
            L->lu[static_cast<size_t>(i) * m + i] = shift + L->A.exit[i];
            for (i64 p = L->A.ptr[i]; p < L->A.ptr[i + 1]; ++p) {
                L->lu[static_cast<size_t>(i) * m + L->A.col[p]] -= L->A.val[p];
            }
        }
        L->piv.resize(m);
        for (int k = 0; k < m; ++k) {
            int p = k;
            for (int i = k + 1; i < m; ++i) {
                if (std::abs(L->lu[static_cast<size_t>(i) * m + k]) > std::abs(L->lu[static_cast<size_t>(p) * m + k])) {
                    p = i;
                }
            }
            L->piv[k] = p;
            for (int j = 0; j < m; ++j) {
                std::swap(L->lu[static_cast<size_t>(k) * m + j], L->lu[static_cast<size_t>(p) * m + j]);
            }
            for (int i = k + 1; i < m; ++i) {
                const double f = L->lu[static_cast<size_t>(i) * m + k] /= L->lu[static_cast<size_t>(k) * m + k];
                for (int j = k + 1; j < m; ++j) {
                    L->lu[static_cast<size_t>(i) * m + j] -= f * L->lu[static_cast<size_t>(k) * m + j];
                }
            }
        }
        return L;
    }
    Grid cg(g.dim, cd, ch);
    std::vector<double> D2 = D;
    for (double &d : D2) {
        d *= 2.0;
    }
    L->coarse = build_level(cg, D2, totals, shift, o, levels_left - 1, C);
    // transfer (multigrid.hpp:50-92)
    std::vector<int> parent(g.V), children(cg.V, 0);
    for (int v = 0; v < g.V; ++v) {
        i64 rem = v, cv = 0, st = 1;
        for (int a = 0; a < g.dim; ++a) {
            i64 c = rem % g.dims[a];
            rem /= g.dims[a];
            if (g.dims[a] > 1) {
                c /= 2;
            }
            cv += c * st;
            st *= cd[a];
        }
        parent[v] = static_cast<int>(cv);
        ++children[cv];
    }
    L->coarse_of.resize(n);
    L->weight.resize(n);
    vec total(L->coarse->space.n, 0.0);
    const int S = L->space.S;
#pragma omp parallel
    {
        std::vector<std::vector<int>> mol;
#pragma omp for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            int k;
            L->space.state(i, k, mol);
            double lw = 0.0;
            std::vector<std::vector<int>> cm(S);
            for (int s = 0; s < S; ++s) {
                std::map<int, int> fine, crs;
                for (int v : mol[s]) {
                    ++fine[v];
                    ++crs[parent[v]];
                    cm[s].push_back(parent[v]);
                }
                for (auto [v, c] : fine) {
                    lw -= std::lgamma(c + 1.0);
                }
                for (auto [a, c] : crs) {
                    lw += std::lgamma(c + 1.0) - c * std::log(double(children[a]));
                }
            }
            L->coarse_of[i] = L->coarse->space.find(cm);
            L->weight[i] = std::exp(lw);
        }
    }
    for (i64 i = 0; i < n; ++i) {
        total[L->coarse_of[i]] += L->weight[i];
    }
    for (i64 i = 0; i < n; ++i) {
        L->weight[i] /= total[L->coarse_of[i]];
    }
    L->crhs.assign(L->coarse->space.n, 0.0);
    L->cx.assign(L->coarse->space.n, 0.0);
    return L;
}

// one cycle from zero (multigrid.hpp:201-228), Jacobi smoothing (:309-317)
void cycle(const Level &L, double shift, const Options &o, const double *b, double *out) {
    const i64 n = L.space.n;
    auto &x = L.x;
    auto &r = L.r;
    auto residual = [&]() {
        L.A.apply(shift, x.data(), r.data());
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            r[i] = b[i] - r[i];
        }
    };
    auto smooth = [&](int sweeps) {
        for (int s = 0; s < sweeps; ++s) {
            residual();
#pragma omp parallel for schedule(static)
            for (i64 i = 0; i < n; ++i) {
                x[i] += o.omega * r[i] / (shift + L.A.exit[i]);
            }
        }
    };
    std::fill(x.begin(), x.end(), 0.0);
    smooth(o.pre);
    residual();
    if (L.coarse) {
        std::fill(L.crhs.begin(), L.crhs.end(), 0.0);
        for (i64 i = 0; i < n; ++i) {
            L.crhs[L.coarse_of[i]] += r[i];
        }
        cycle(*L.coarse, shift, o, L.crhs.data(), L.cx.data());
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            x[i] += L.weight[i] * L.cx[L.coarse_of[i]];
        }
    } else {
        const int m = static_cast<int>(n);
        std::vector<double> y(r.begin(), r.end());
        for (int k = 0; k < m; ++k) {
            std::swap(y[k], y[L.piv[k]]);
        }
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < i; ++j) {
                y[i] -= L.lu[static_cast<size_t>(i) * m + j] * y[j];
            }
        }
        for (int i = m - 1; i >= 0; --i) {
            for (int j = i + 1; j < m; ++j) {
                y[i] -= L.lu[static_cast<size_t>(i) * m + j] * y[j];
            }
            y[i] /= L.lu[static_cast<size_t>(i) * m + i];
        }
        for (i64 i = 0; i < n; ++i) {
            x[i] += y[i];
        }
    }
    smooth(o.post);
    std::copy(x.begin(), x.end(), out);
}

// ---- GMRES (right preconditioned, MGS, Givens) ---------------------------------------------
struct Result {
    i64 iterations = 0;
    double residual = 0;
    bool converged = false;
};

double dot(const vec &a, const vec &b) {
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (size_t i = 0; i < a.size(); ++i) {
        s += a[i] * b[i];
    }
    return s;
}

template <typename ApplyA, typename ApplyM>
Result gmres(ApplyA &&A, ApplyM &&M, const vec &b, vec &x, double tol, i64 maxit, int restart) {
    const i64 n = static_cast<i64>(b.size());
    const int m = static_cast<int>(std::min<i64>(restart, n));
    Result res;
    vec r(n), w(n), z(n);
    auto true_res = [&]() {
        A(x.data(), w.data());
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            r[i] = b[i] - w[i];
        }
        return std::sqrt(dot(r, r));
    };
    double beta = true_res();
    res.residual = beta;
    if (beta <= tol) {
        res.converged = true;
        return res;
    }
    std::vector<vec> V(m + 1, vec(n));
    std::vector<vec> H(m + 1, vec(m, 0.0));
    vec cs(m), sn(m), g(m + 1), y(m);
    while (res.iterations < maxit) {
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) {
            V[0][i] = r[i] / beta;
        }
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        for (int j = 0; j < m && res.iterations < maxit; ++j) {
            M(V[j].data(), z.data());
            A(z.data(), w.data());
            for (int i = 0; i <= j; ++i) {
                H[i][j] = dot(w, V[i]);
                const double hij = H[i][j];
#pragma omp parallel for schedule(static)
                for (i64 t = 0; t < n; ++t) {
                    w[t] -= hij * V[i][t];
                }
            }
            const double h = std::sqrt(dot(w, w));
            H[j + 1][j] = h;
            for (int i = 0; i < j; ++i) {
                const double a = H[i][j], c = H[i + 1][j];
                H[i][j] = cs[i] * a + sn[i] * c;
                H[i + 1][j] = -sn[i] * a + cs[i] * c;
            }
            const double a = H[j][j], c = H[j + 1][j], den = std::hypot(a, c);
            cs[j] = den > 0 ? a / den : 1.0;
            sn[j] = den > 0 ? c / den : 0.0;
            H[j][j] = den;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++res.iterations;
            k = j + 1;
            if (std::abs(g[j + 1]) <= tol || !(h > 0)) {
                break;
            }
#pragma omp parallel for schedule(static)
            for (i64 t = 0; t < n; ++t) {
                V[j + 1][t] = w[t] / h;
            }
        }
        for (int i = k - 1; i >= 0; --i) {
            double s = g[i];
            for (int t = i + 1; t < k; ++t) {
                s -= H[i][t] * y[t];
            }
            y[i] = s / H[i][i];
        }
        std::fill(w.begin(), w.end(), 0.0);
        for (int j = 0; j < k; ++j) {
#pragma omp parallel for schedule(static)
            for (i64 t = 0; t < n; ++t) {
                w[t] += y[j] * V[j][t];
            }
        }
        M(w.data(), z.data());
#pragma omp parallel for schedule(static)
        for (i64 t = 0; t < n; ++t) {
            x[t] += z[t];
        }
        beta = true_res();
        res.residual = beta;
        if (beta <= tol) {
            res.converged = true;
            return res;
        }
    }
    return res;
}

// ---- driver --------------------------------------------------------------------------------
std::map<std::string, std::string> kv;
std::string get(const std::string &k, const std::string &d) {
    auto it = kv.find(k);
    return it == kv.end() ? d : it->second;
}
double num(const std::string &k, double d) { return kv.count(k) ? std::stod(kv[k]) : d; }

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace

int main(int argc, char **argv) {
    for (int i = 1; i < argc; ++i) {
        std::string s(argv[i]);
        const auto eq = s.find('=');
        if (eq == std::string::npos) {
            std::cerr << "expected key=value\n";
            return 2;
        }
        kv[s.substr(0, eq)] = s.substr(eq + 1);
    }
    if (kv.count("threads")) {
        omp_set_num_threads(std::stoi(kv["threads"]));
    }
    try {
        const int dim = static_cast<int>(num("dim", 1));
        const i64 cells = static_cast<i64>(num("cells", 16));
        i64 dims[3] = {1, 1, 1};
        double h[3] = {1, 1, 1};
        for (int a = 0; a < dim; ++a) {
            dims[a] = cells;
            h[a] = num("h", 1.0 / static_cast<double>(cells));
        }
        const Grid grid(dim, dims, h);
        const std::string model = get("model", "birth_death");
        std::vector<double> D;
        std::vector<Reaction> rx;
        const double birth = num("birth", 0.05), death = num("death", 0.02), k = num("k", 10.0);
        if (model == "birth_death") {
            D = {num("D", 1.0)};
            rx.push_back({{1}, [=](const std::vector<int> &, double vol) { return birth * vol; }});
            rx.push_back({{-1}, [=](const std::vector<int> &n, double) { return death * n[0]; }});
        } else if (model == "annihilation") {
            D = {num("D", 1.0), num("D2", num("D", 1.0))};
            rx.push_back({{-1, -1}, [=](const std::vector<int> &n, double vol) {
                              return k * n[0] * n[1] / vol;
                          }});
        } else {
            D = {num("D", 1.0)};
        }
        std::vector<int> caps;
        {
            std::stringstream ss(get("cap", "3"));
            std::string item;
            while (std::getline(ss, item, ',')) {
                caps.push_back(std::stoi(item));
            }
        }
        const int S = static_cast<int>(caps.size());
        const int tmax = *std::max_element(caps.begin(), caps.end());
        const Choose C(tmax + 1, grid.V + tmax + 2);
        const double shift = num("shift", 0.5);
        const Options o;

        auto t0 = std::chrono::steady_clock::now();
        Space box;
        box.V = grid.V;
        box.S = S;
        box.C = &C;
        std::vector<int> t(S, 0);
        while (true) {
            box.add(t);
            int s = S - 1;
            while (s >= 0 && t[s] == caps[s]) {
                t[s] = 0;
                --s;
            }
            if (s < 0) {
                break;
            }
            ++t[s];
        }
        Operator A;
        A.build(box, grid, D, rx, get("boundary", "absorbing") == "absorbing");
        std::vector<std::unique_ptr<Level>> mg;
        for (const Sector &sec : box.sectors) {
            mg.push_back(build_level(grid, D, sec.totals, shift, o, o.max_levels, C));
        }
        const double setup_ms = ms_since(t0);
        const i64 N = box.n;

        vec b;
        const std::string rhs = get("rhs", "uniform");
        const auto seed = static_cast<std::uint64_t>(num("seed", 0));
        if (rhs == "uniform") {
            b = oracle::uniform_rhs(seed, N);
        } else if (rhs == "dirichlet") {
            b = oracle::dirichlet_rhs(seed, N);
        } else {
            b.resize(N);
            std::ifstream f(rhs, std::ios::binary);
            f.read(reinterpret_cast<char *>(b.data()), static_cast<std::streamsize>(N * 8));
        }
        auto applyA = [&](const double *x, double *y) { A.apply(shift, x, y); };
        auto applyM = [&](const double *v, double *z) {
            for (size_t s = 0; s < box.sectors.size(); ++s) {
                const Sector &sec = box.sectors[s];
                cycle(*mg[s], shift, o, v + sec.begin, z + sec.begin);
            }
        };
        const double bnorm = std::sqrt(dot(b, b));
        const double tol = num("tol", 1e-10) * bnorm;
        const int restart = static_cast<int>(num("restart", 30));
        const i64 maxit = static_cast<i64>(num("maxit", 1000));
        const i64 sample = static_cast<i64>(num("sample_iters", 0));
        const int warmup = static_cast<int>(num("warmup", 0)), solves = static_cast<int>(num("solves", 1));
        vec x(N, 0.0);
        Result r;
        std::vector<double> times;
        i64 full_iterations = -1; // iterations of the first solve run to convergence
        for (int s = 0; s < warmup + solves; ++s) {
            std::fill(x.begin(), x.end(), 0.0);
            t0 = std::chrono::steady_clock::now();
            const bool sampled = sample > 0 && s >= warmup;
            r = gmres(applyA, applyM, b, x, tol, sampled ? sample : maxit, restart);
            if (!sampled && full_iterations < 0) {
                full_iterations = r.iterations;
            }
            if (s >= warmup) {
                times.push_back(ms_since(t0));
            }
        }
        vec w(N);
        applyA(x.data(), w.data());
        double rn = 0;
        for (i64 i = 0; i < N; ++i) {
            rn += (b[i] - w[i]) * (b[i] - w[i]);
        }
        std::ostringstream out;
        out.precision(17);
        out << "{\"N\":" << N << ",\"threads\":" << omp_get_max_threads() << ",\"setup_ms\":" << setup_ms
            << ",\"iterations\":" << r.iterations << ",\"full_iterations\":" << full_iterations
            << ",\"converged\":" << r.converged
            << ",\"true_rel_residual\":" << std::sqrt(rn) / bnorm << ",\"solve_ms\":[";
        for (size_t i = 0; i < times.size(); ++i) {
            out << (i ? "," : "") << times[i];
        }
        out << "]}";
        const std::string dir = get("out", "");
        if (!dir.empty()) {
            std::ofstream f(dir + "/x_port.f64", std::ios::binary);
            f.write(reinterpret_cast<const char *>(x.data()), static_cast<std::streamsize>(N * 8));
        }
        std::cout << out.str() << std::endl;
    } catch (const std::exception &e) {
        std::cerr << "mf_port: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
