// Host side of the B200 resolvent engine (see engine.hpp).
#include "engine.hpp"
#include "dense_inverse.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <map>
#include <numeric>

namespace mkb {

void check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) {
        return;
    }
    const int code = (e == cudaErrorMemoryAllocation) ? kENoMem : kECuda;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------
// binomials and spaces

std::unique_ptr<Space> Space::make(int V, const std::vector<int> &limits, bool is_box) {
    const int S = static_cast<int>(limits.size());
    if (V < 1 || S < 1) {
        throw Error(kEInval, "population state space needs a voxel and a species");
    }
    if (S > kMaxSpecies) {
        throw Error(kEInval, "at most 4 species are supported");
    }
    for (int t : limits) {
        if (t < 0) {
            throw Error(kEInval, "species totals must be nonnegative");
        }
        if (t > kHostIndexCap) {
            throw Error(kEInval, "species totals above 1024 are not supported");
        }
    }
    auto sp = std::make_unique<Space>();
    sp->V = V;
    sp->S = S;
    sp->is_box = is_box;
    sp->limits = limits;
    sp->max_total = *std::max_element(limits.begin(), limits.end());
    sp->max_mol = std::accumulate(limits.begin(), limits.end(), 0);
    sp->binom = std::make_shared<Binomials>(sp->max_total + 1, V + sp->max_total + 1);
    const std::vector<std::vector<int>> totals =
        is_box ? box_totals(limits) : std::vector<std::vector<int>>{limits};
    sp->sectors = layout_sectors(V, S, totals, sp->binom->host_view(), &sp->n);
    sp->d_sectors.upload(sp->sectors);
    sp->d_limits.upload(limits);
    return sp;
}

int Space::find_sector(const int *totals) const {
    if (!is_box) {
        for (int s = 0; s < S; ++s) {
            if (totals[s] != limits[s]) {
                return -1;
            }
        }
        return 0;
    }
    int k = 0;
    for (int s = 0; s < S; ++s) {
        if (totals[s] < 0 || totals[s] > limits[s]) {
            return -1;
        }
        k = k * (limits[s] + 1) + totals[s];
    }
    return k;
}

int Space::sector_of(std::int64_t i) const {
    auto it = std::upper_bound(sectors.begin(), sectors.end(), i,
                               [](std::int64_t v, const SectorDesc &s) { return v < s.begin; });
    return static_cast<int>(it - sectors.begin()) - 1;
}

std::int64_t Space::rank(const int *state) const {
    int totals[kMaxSpecies] = {};
    for (int v = 0; v < V; ++v) {
        for (int s = 0; s < S; ++s) {
            const int c = state[static_cast<std::int64_t>(v) * S + s];
            if (c < 0) {
                return -1;
            }
            totals[s] += c;
        }
    }
    const int k = find_sector(totals);
    if (k < 0) {
        return -1;
    }
    const SectorDesc &sec = sectors[k];
    const BinomTable B = binom->host_view();
    std::vector<int> buf(kHostIndexCap);
    auto &u = *reinterpret_cast<int(*)[kHostIndexCap]>(buf.data());
    std::int64_t local = 0;
    for (int s = 0; s < S; ++s) {
        int n = 0;
        for (int v = V - 1; v >= 0; --v) {
            for (int q = 0; q < state[static_cast<std::int64_t>(v) * S + s]; ++q) {
                u[n++] = V - 1 - v;
            }
        }
        local += rank_species<kHostIndexCap>(B, u, n) * sec.stride[s];
    }
    return sec.begin + local;
}

void Space::unrank(std::int64_t i, int *state) const {
    std::fill(state, state + static_cast<std::int64_t>(V) * S, 0);
    if (i < 0 || i >= n) {
        throw Error(kEInval, "state index out of range");
    }
    const SectorDesc &sec = sectors[sector_of(i)];
    std::int64_t rank[kMaxSpecies];
    split_local(sec, S, i - sec.begin, rank);
    std::vector<int> buf(kHostIndexCap);
    auto &u = *reinterpret_cast<int(*)[kHostIndexCap]>(buf.data());
    const BinomTable B = binom->host_view();
    for (int s = 0; s < S; ++s) {
        unrank_species<kHostIndexCap>(B, rank[s], sec.total[s], V, u);
        for (int p = 0; p < sec.total[s]; ++p) {
            ++state[static_cast<std::int64_t>(V - 1 - u[p]) * S + s];
        }
    }
}

// ---------------------------------------------------------------------------------------
// models

template <typename T>
void ModelTables<T>::build(const Model &m, double diff_scale, bool with_reactions, bool absorbing) {
    h.build(m, diff_scale, with_reactions, absorbing);
    nbr_ptr.upload(h.nbr_ptr);
    nbr_idx.upload(h.nbr_idx);
    in_coef.upload(h.in_coef);
    deg_coef.upload(h.deg_coef);
    vparity.upload(h.vparity);
    vmask.upload(h.vmask);
    vclass.upload(h.vclass);
    rate.upload(h.rate);
    host = h.view;
    dev = h.view;
    dev.nbr_ptr = nbr_ptr.get();
    dev.nbr_idx = nbr_idx.get();
    dev.in_coef = in_coef.get();
    dev.deg_coef = deg_coef.get();
    dev.vparity = vparity.get();
    dev.vmask = h.vmask.empty() ? nullptr : vmask.get();
    dev.vclass = h.vclass.empty() ? nullptr : vclass.get();
    dev.rate = h.rate.empty() ? nullptr : rate.get();
}

template struct ModelTables<double>;
template struct ModelTables<float>;

// ---------------------------------------------------------------------------------------
// operator levels and the generator

namespace {
std::atomic<int> g_row_path{0};
} // namespace

void set_row_path(int path) { g_row_path.store(path == 1 || path == 2 ? path : 0); }
int row_path() { return g_row_path.load(); }

void OperatorLevel::finalize(const Model &m, bool with_reactions) {
    if (n >= (std::int64_t(1) << 31)) {
        throw Error(kEInval, "state spaces of 2^31 states or more are not supported on the device");
    }
    mol_cap = mol_cap_for(S, max_species_total(sectors));
    if (mol_cap < 0) {
        throw Error(kEInval, "more than 64 molecules of one species per state are not supported");
    }
    couple_sectors<double>(sectors, S, m, t64.host, with_reactions);
    tiles.clear();
    for (std::size_t k = 0; k < sectors.size(); ++k) {
        const SectorDesc &sec = sectors[k];
        // heavy rows: a warp each, or a whole block each when warps alone would fill less than
        // about two waves of the GPU while each lane loops over many voxels
        const bool few = sec.size <= 4 * 148 || (sec.size * 32 <= 2 * 148 * 2048 && V >= 1024);
        const int kind = sec.heavy ? (few ? 2 : 1) : 0;
        const int rows = kind == 0 ? kRowBlock : (kind == 1 ? kWarpRows : 1);
        for (std::int64_t l = 0; l < sec.size; l += rows) {
            Tile t;
            t.local0 = l;
            t.sector = static_cast<int>(k);
            t.kind = kind;
            t.count = static_cast<int>(std::min<std::int64_t>(rows, sec.size - l));
            tiles.push_back(t);
        }
    }
    if (tiles.size() > 0x7fffffffULL) {
        throw Error(kEInval, "space too large for one launch");
    }
    // rows the stencil kernels serve: light rows of a structured grid with per-voxel masks; in
    // the pair and single-molecule shapes, only sectors whose reactions their tables cover
    stencil_tiles.clear();
    general_tiles.clear();
    std::vector<StencilSector<float>> h_ss32;
    std::vector<double> h_ddeg64;
    std::vector<float> h_ddeg32;
    const bool pair = build_stencil_tables<double>(sectors, S, mol_cap, t64.h.view, t64.h.rate,
                                                   t64.h.deg_coef, h_ss64, h_ddeg64, sv64);
    build_stencil_tables<float>(sectors, S, mol_cap, t64.h.view, t64.h.rate, t64.h.deg_coef, h_ss32,
                                h_ddeg32, sv32);
    heavy_tiles.clear();
    general_rest.clear();
    if (t64.host.grid_dim > 0 && !t64.h.vmask.empty() && stencil_shape(S, mol_cap)) {
        for (const Tile &t : tiles) {
            const bool light = t.kind == 0 && !sectors[t.sector].heavy;
            const bool served = light && (!pair || h_ss64[t.sector].fast);
            (served ? stencil_tiles : general_tiles).push_back(t);
            if (!served) {
                const bool heavy = pair && !light && h_ss64[t.sector].fast && h_ss64[t.sector].heavy_ok;
                (heavy ? heavy_tiles : general_rest).push_back(t);
            }
        }
        if (stencil_tiles.empty()) {
            general_tiles.clear();
            heavy_tiles.clear();
            general_rest.clear();
        }
    }
    // sectors of every pair u0 <= u1 of the V voxels: the pair-strip form, a tile per pair of
    // triangle rows. On grids of fewer voxels a level's rows fit a few waves of one launch, and
    // a second launch per pass would cost more than the form saves.
    strip_tiles.clear();
    stencil_rest.clear();
    constexpr int kStripMinVoxels = 1024;
    if (pair && S == 1 && !stencil_tiles.empty() && V >= kStripMinVoxels) {
        const std::int64_t pairs = static_cast<std::int64_t>(V) * (V + 1) / 2;
        std::vector<char> strip(sectors.size(), 0);
        for (std::size_t k = 0; k < sectors.size(); ++k) {
            const SectorDesc &sec = sectors[k];
            strip[k] = !sec.heavy && h_ss64[k].fast && h_ss64[k].total[0] == 2 && sec.size == pairs ? 1 : 0;
            for (int q = 0; strip[k] && q < (V + 1) / 2; ++q) {
                Tile t;
                t.local0 = q;
                t.sector = static_cast<int>(k);
                t.kind = 3;
                strip_tiles.push_back(t);
            }
        }
        for (const Tile &t : stencil_tiles) {
            if (!strip[t.sector]) {
                stencil_rest.push_back(t);
            }
        }
    }
    d_strip_tiles.upload(strip_tiles);
    d_stencil_rest.upload(stencil_rest);
    // heavy rows of one molecule fed by the pair sector: groups of eight rows
    heavy_group_tiles.clear();
    if (pair && S == 1 && !heavy_tiles.empty()) {
        std::vector<char> grouped(sectors.size(), 0);
        for (std::size_t k = 0; k < sectors.size(); ++k) {
            const StencilSector<double> &ss = h_ss64[k];
            bool ok = sectors[k].heavy && ss.fast && ss.heavy_ok && ss.total[0] == 1 && ss.n_heavy > 0 &&
                      sectors[k].size == V;
            for (int q = 0; ok && q < ss.n_heavy; ++q) {
                ok = ss.heavy_copies[q] == 1;
            }
            grouped[k] = ok ? 1 : 0;
            for (std::int64_t l = 0; ok && l < sectors[k].size; l += kHeavyGroupRows) {
                Tile t;
                t.local0 = l;
                t.sector = static_cast<int>(k);
                t.kind = 4;
                t.count = static_cast<int>(std::min<std::int64_t>(kHeavyGroupRows, sectors[k].size - l));
                heavy_group_tiles.push_back(t);
            }
        }
        std::vector<Tile> rest;
        for (const Tile &t : heavy_tiles) {
            if (!grouped[t.sector]) {
                rest.push_back(t);
            }
        }
        heavy_tiles.swap(rest);
    }
    d_heavy_group_tiles.upload(heavy_group_tiles);
    d_heavy_tiles.upload(heavy_tiles);
    d_general_rest.upload(general_rest);
    ss64.upload(h_ss64);
    ss32.upload(h_ss32);
    ddeg64.upload(h_ddeg64);
    ddeg32.upload(h_ddeg32);
    sv64.sectors = pair ? ss64.get() : nullptr;
    sv64.ddeg = pair ? ddeg64.get() : nullptr;
    sv32.sectors = pair ? ss32.get() : nullptr;
    sv32.ddeg = pair ? ddeg32.get() : nullptr;
    d_sectors.upload(sectors);
    d_tiles.upload(tiles);
    d_stencil_tiles.upload(stencil_tiles);
    d_general_tiles.upload(general_tiles);
}

template <typename T>
RowParams<T> OperatorLevel::params() const {
    RowParams<T> p;
    p.B = binom->device_view();
    p.sectors = d_sectors.get();
    p.tiles = d_tiles.get();
    if constexpr (std::is_same_v<T, double>) {
        p.md = t64.dev;
        p.sv = sv64;
    } else {
        p.md = t32.dev;
        p.sv = sv32;
    }
    p.n_tiles = static_cast<int>(tiles.size());
    return p;
}

template <typename T>
void OperatorLevel::run(RowMode mode, const RowParams<T> &p, cudaStream_t stream) const {
    if (stencil_tiles.empty() || !stencil_mode(mode) || row_path() == 1) {
        check_cuda(launch_rows<T>(mode, S, mol_cap, p, stream), "row kernel launch");
        return;
    }
    RowParams<T> q = p;
    q.mode = mode;
    if ((!heavy_tiles.empty() || !heavy_group_tiles.empty()) && pair_heavy_mode(mode)) {
        // rows with in-jumps from every voxel first (they read the whole next sector), then the rest
        cudaError_t e = cudaSuccess;
        if (!heavy_group_tiles.empty()) {
            q.tiles = d_heavy_group_tiles.get();
            q.n_tiles = static_cast<int>(heavy_group_tiles.size());
            if constexpr (std::is_same_v<T, double>) {
                e = launch_pair_heavy_group_rows_f64(q, stream);
            } else {
                e = launch_pair_heavy_group_rows_f32(q, stream);
            }
            check_cuda(e, "pair heavy group kernel launch");
        }
        if (!heavy_tiles.empty()) {
            q.tiles = d_heavy_tiles.get();
            q.n_tiles = static_cast<int>(heavy_tiles.size());
            if constexpr (std::is_same_v<T, double>) {
                e = launch_pair_heavy_rows_f64(q, stream);
            } else {
                e = launch_pair_heavy_rows_f32(q, stream);
            }
            check_cuda(e, "pair heavy row kernel launch");
        }
        if (!general_rest.empty()) {
            q.tiles = d_general_rest.get();
            q.n_tiles = static_cast<int>(general_rest.size());
            check_cuda(launch_rows<T>(mode, S, mol_cap, q, stream), "row kernel launch");
        }
    } else if (!general_tiles.empty()) {
        q.tiles = d_general_tiles.get();
        q.n_tiles = static_cast<int>(general_tiles.size());
        check_cuda(launch_rows<T>(mode, S, mol_cap, q, stream), "row kernel launch");
    }
    const bool strip = !strip_tiles.empty() && row_path() == 0;
    if (strip) {
        q.tiles = d_strip_tiles.get();
        q.n_tiles = static_cast<int>(strip_tiles.size());
        cudaError_t e;
        if constexpr (std::is_same_v<T, double>) {
            e = launch_pair_strip_rows_f64(q, stream);
        } else {
            e = launch_pair_strip_rows_f32(q, stream);
        }
        check_cuda(e, "pair strip row kernel launch");
        if (stencil_rest.empty()) {
            return;
        }
    }
    q.tiles = strip ? d_stencil_rest.get() : d_stencil_tiles.get();
    q.n_tiles = static_cast<int>(strip ? stencil_rest.size() : stencil_tiles.size());
    cudaError_t e;
    if constexpr (std::is_same_v<T, double>) {
        e = launch_stencil_rows_f64(q, S, mol_cap, stream);
    } else {
        e = launch_stencil_rows_f32(q, S, mol_cap, stream);
    }
    check_cuda(e, "stencil row kernel launch");
}

template RowParams<double> OperatorLevel::params<double>() const;
template RowParams<float> OperatorLevel::params<float>() const;
template void OperatorLevel::run<double>(RowMode, const RowParams<double> &, cudaStream_t) const;
template void OperatorLevel::run<float>(RowMode, const RowParams<float> &, cudaStream_t) const;

Generator::Generator(const Space &sp, const Model &model, bool absorbing_)
    : space(&sp), absorbing(absorbing_) {
    model.validate();
    if (model.V != sp.V || model.S != sp.S) {
        throw Error(kEInval, "model and space disagree on voxels or species");
    }
    if (model.R > 0) {
        for (int s = 0; s < sp.S; ++s) {
            if (model.tmax[s] < sp.limits[s]) {
                throw Error(kEInval, "reaction rates must be tabulated up to the space's totals");
            }
        }
    }
    op.V = sp.V;
    op.S = sp.S;
    op.n = sp.n;
    op.sectors = sp.sectors;
    op.binom = sp.binom;
    op.t64.build(model, 1.0, true, absorbing);
    op.t32.build(model, 1.0, true, absorbing);
    op.finalize(model, true);
}

template <typename T>
void Generator::apply(RowMode mode, T shift, const T *x, const T *b, T *y, T *aux,
                      cudaStream_t stream, int nb, std::int64_t ld) const {
    RowParams<T> p = op.params<T>();
    p.shift = shift;
    p.x = x;
    p.b = b;
    p.y = y;
    p.aux = aux;
    p.nb = nb;
    p.ldv = ld;
    op.run<T>(mode, p, stream);
}

template void Generator::apply<double>(RowMode, double, const double *, const double *, double *,
                                       double *, cudaStream_t, int, std::int64_t) const;
template void Generator::apply<float>(RowMode, float, const float *, const float *, float *,
                                      float *, cudaStream_t, int, std::int64_t) const;

// ---------------------------------------------------------------------------------------
// multigrid

namespace {

template <typename T>
__global__ void axpy_t_kernel(T a, const T *x, T *y, std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        y[i] += a * x[i];
    }
}

template <typename T>
void axpy_t(T a, const T *x, T *y, std::int64_t n, cudaStream_t stream) {
    if (n == 0) {
        return;
    }
    const std::int64_t want = (n + 255) / 256;
    const auto blocks = static_cast<unsigned>(std::min<std::int64_t>(want, 148 * 8));
    count_launches(1);
    axpy_t_kernel<T><<<blocks, 256, 0, stream>>>(a, x, y, n);
    check_cuda(cudaGetLastError(), "axpy");
}

// a whole level (every sector, reactions included) as one dense block, from the same
// matrix-free rows (host, generic shape)
void assemble_level(const OperatorLevel &op, double shift, std::vector<double> &A) {
    const auto n = static_cast<std::size_t>(op.n);
    A.assign(n * n, 0.0);
    const BinomTable B = op.binom->host_view();
    auto st = std::make_unique<RowState<kMaxSpecies, 64>>();
    for (const SectorDesc &sec : op.sectors) {
        for (std::int64_t i = 0; i < sec.size; ++i) {
            load_state<kMaxSpecies, 64>(B, sec, op.S, op.V, i, *st);
            double exit = 0.0, leak = 0.0;
            const std::size_t row = static_cast<std::size_t>(sec.begin + i);
            visit_row<double, kMaxSpecies, 64>(B, op.sectors.data(), sec, op.t64.host, i, *st, true, 0,
                                               1, exit, leak, [&](std::int64_t j, double a, double) {
                                                   A[row * n + static_cast<std::size_t>(j)] -= a;
                                               });
            A[row * n + row] += shift + exit;
        }
    }
}

// the terminal block of one sector, dense, from the same matrix-free rows (host, generic shape)
void assemble_terminal(const OperatorLevel &op, int slot, double shift, std::vector<double> &A) {
    const SectorDesc &sec = op.sectors[slot];
    const auto n = static_cast<int>(sec.size);
    A.assign(static_cast<std::size_t>(n) * n, 0.0);
    const BinomTable B = op.binom->host_view();
    auto st = std::make_unique<RowState<kMaxSpecies, 64>>();
    for (int i = 0; i < n; ++i) {
        load_state<kMaxSpecies, 64>(B, sec, op.S, op.V, i, *st);
        double exit = 0.0, leak = 0.0;
        visit_row<double, kMaxSpecies, 64>(B, op.sectors.data(), sec, op.t64.host, i, *st, true, 0, 1, exit,
                                leak, [&](std::int64_t j, double a, double) {
                                    A[static_cast<std::size_t>(i) * n + (j - sec.begin)] -= a;
                                });
        A[static_cast<std::size_t>(i) * n + i] += shift + exit;
    }
}

} // namespace

namespace {
const Model &fine_model(const std::vector<const Model *> &level_models) {
    if (level_models.empty() || !level_models[0]) {
        throw Error(kEInval, "full-operator multigrid: no level models");
    }
    return *level_models[0];
}
} // namespace

Multigrid::Multigrid(const Space &space, const std::vector<const Model *> &level_models,
                     double shift_, const MultigridOptions &o)
    : Multigrid(space, fine_model(level_models), shift_, o, &level_models) {}

Multigrid::Multigrid(const Space &space, const Model &model, double shift_,
                     const MultigridOptions &o)
    : Multigrid(space, model, shift_, o, nullptr) {}

Multigrid::Multigrid(const Space &space, const Model &model, double shift_,
                     const MultigridOptions &o, const std::vector<const Model *> *level_models)
    : Preconditioner(space.n), opt(o), shift(shift_), full_(level_models != nullptr),
      binom(space.binom) {
    if (!(shift > 0.0)) {
        throw Error(kEInval, "population_multigrid: shift must be positive");
    }
    model.validate();
    if (!model.has_grid) {
        throw Error(kEInval, "sector_multigrid needs a structured grid");
    }
    if (model.V != space.V || model.S != space.S) {
        throw Error(kEInval, "model and space disagree on voxels or species");
    }
    if (opt.smoother < 0 || opt.smoother > 3 || opt.precision < 0 || opt.precision > 1) {
        throw Error(kEInval, "unknown smoother or precision");
    }
    if (opt.smoother == 3 && opt.batch != 1) {
        throw Error(kEInval, "the aggregate-block smoother serves one right-hand side at a time");
    }
    if (full_ && opt.smoother != 0 && opt.smoother != 1) {
        throw Error(kEInval, "the full-operator multigrid smooths by weighted Jacobi (0) or "
                             "multicolour Gauss-Seidel (1)");
    }
    if (opt.cycle_type != 0 && (opt.cycle_type != 1 || !full_ || opt.precision != 0 || opt.batch != 1)) {
        throw Error(kEInval, "the K-cycle belongs to the full-operator multigrid, in FP64, one "
                             "right-hand side at a time");
    }
    if (opt.batch < 1 || opt.batch > kRowBatch) {
        throw Error(kEInval, "multigrid batch must be in 1.." + std::to_string(kRowBatch));
    }
    const int S = space.S;
    std::vector<double> h_lgf(space.max_total + 2);
    for (std::size_t k = 0; k < h_lgf.size(); ++k) {
        h_lgf[k] = std::lgamma(static_cast<double>(k) + 1.0);
    }
    lgf.upload(h_lgf);

    // depth 0: every sector of the space, on the model's own grid
    std::vector<std::vector<int>> totals;
    std::vector<int> box_of;
    for (std::size_t k = 0; k < space.sectors.size(); ++k) {
        totals.emplace_back(space.sectors[k].total, space.sectors[k].total + S);
        box_of.push_back(static_cast<int>(k));
    }
    std::int64_t dims[3] = {model.dims[0], model.dims[1], model.dims[2]};
    double spacing[3] = {model.spacing[0], model.spacing[1], model.spacing[2]};
    double scale = 1.0;
    for (int d = 0; !totals.empty(); ++d) {
        auto L = std::make_unique<Level>();
        auto grid_model = Model::grid(model.dim, dims, spacing, model.diff);
        if (full_) {
            // this level's reactions, tabulated by the caller at its voxel volume
            if (d >= static_cast<int>(level_models->size()) || !(*level_models)[d]) {
                throw Error(kEInval, "full-operator multigrid: no model for level " + std::to_string(d));
            }
            const Model &lm = *(*level_models)[d];
            if (lm.V != grid_model->V || lm.S != S) {
                throw Error(kEInval, "full-operator multigrid: level " + std::to_string(d) +
                                         "'s model is not on the coarsened grid");
            }
            grid_model->R = lm.R;
            grid_model->change = lm.change;
            grid_model->tmax = lm.tmax;
            grid_model->nvc = lm.nvc;
            grid_model->vclass = lm.vclass;
            grid_model->rates = lm.rates;
            grid_model->validate();
        }
        L->op.V = grid_model->V;
        L->op.S = S;
        L->op.binom = binom;
        L->op.sectors = layout_sectors(grid_model->V, S, totals, binom->host_view(), &L->op.n);
        L->op.t64.build(*grid_model, scale, full_, true);
        L->op.t32.build(*grid_model, scale, full_, true);
        L->pre = opt.pre_sweeps + d * opt.sweep_growth;
        L->post = opt.post_sweeps + d * opt.sweep_growth;
        L->box_sector = box_of;

        // coarsen (markovkit/rdme/multigrid.hpp:25-42)
        std::int64_t cdims[3];
        double cspacing[3];
        const bool can_coarsen = coarsen_grid(model.dim, dims, spacing, cdims, cspacing);
        const int levels_left = opt.max_levels - d;

        std::vector<std::vector<int>> next_totals;
        std::vector<int> next_box;
        // the full operator couples the sectors: the level coarsens or stops as a whole
        const bool whole_terminal = full_ && (L->op.n <= opt.coarsest_size || levels_left <= 1 ||
                                              !can_coarsen ||
                                              d + 1 >= static_cast<int>(level_models->size()));
        if (whole_terminal) {
            if (L->op.n > 8192) {
                throw Error(kEInval, "full-operator multigrid: coarsest level larger than 8192 states");
            }
            TerminalBlock tb;
            tb.begin = 0;
            tb.n = static_cast<int>(L->op.n);
            L->h_term.push_back(tb);
        }
        for (std::size_t k = 0; k < totals.size(); ++k) {
            SectorDesc &sec = L->op.sectors[k];
            if (full_) {
                if (!whole_terminal) {
                    sec.coarse = static_cast<int>(next_totals.size());
                    next_totals.push_back(totals[k]);
                    next_box.push_back(box_of[k]);
                }
                continue;
            }
            const bool terminal =
                sec.size <= opt.coarsest_size || levels_left <= 1 || !can_coarsen;
            if (terminal) {
                sec.terminal = static_cast<int>(L->h_term.size());
                TerminalBlock tb;
                tb.begin = sec.begin;
                tb.n = static_cast<int>(sec.size);
                if (sec.size > 8192) {
                    throw Error(kEInval, "terminal multigrid block larger than 8192 states");
                }
                L->h_term.push_back(tb);
            } else {
                sec.coarse = static_cast<int>(next_totals.size());
                next_totals.push_back(totals[k]);
                next_box.push_back(box_of[k]);
            }
        }
        L->op.finalize(*grid_model, full_);
        if (full_) {
            // Gauss-Seidel colour classes of the sectors: a greedy colouring of the graph whose
            // edges are the reactions between sectors, so that no in-jump of a class's rows
            // starts in the same class; with the checkerboard colour inside a sector (every
            // diffusion jump flips it) no pass reads what it writes
            auto &secs = L->op.sectors;
            for (std::size_t k = 0; k < secs.size(); ++k) {
                std::vector<bool> used(secs.size() + 1, false);
                for (int r = 0; r < grid_model->R; ++r) {
                    for (int nb : {secs[k].src[r], secs[k].dst[r]}) {
                        if (nb >= 0 && static_cast<std::size_t>(nb) < k) {
                            used[static_cast<std::size_t>(secs[nb].gs_class)] = true;
                        }
                    }
                }
                int c = 0;
                while (used[static_cast<std::size_t>(c)]) {
                    ++c;
                }
                secs[k].gs_class = c;
                L->n_classes = std::max(L->n_classes, c + 1);
            }
            L->op.d_sectors.upload(secs);
        }

        // dense inverses of the terminal blocks, from the same matrix-free rows, all of a level
        // at once (on the device when they are large)
        std::vector<double> inv_all, A, A_all, dense_all;
        std::vector<std::int64_t> term_offset;
        std::vector<int> term_n;
        if (whole_terminal) {
            assemble_level(L->op, shift, A_all);
            term_offset.push_back(0);
            term_n.push_back(static_cast<int>(L->op.n));
        }
        for (std::size_t k = 0; k < L->op.sectors.size() && !full_; ++k) {
            const SectorDesc &sec = L->op.sectors[k];
            if (sec.terminal < 0) {
                continue;
            }
            assemble_terminal(L->op, static_cast<int>(k), shift, A);
            if (opt.smoother == 3) {
                DenseBlock db;
                db.begin = sec.begin;
                db.a_offset = static_cast<std::int64_t>(dense_all.size());
                db.n = static_cast<int>(sec.size);
                L->h_dense.push_back(db);
                dense_all.insert(dense_all.end(), A.begin(), A.end());
            }
            L->h_term[sec.terminal].inv_offset = static_cast<std::int64_t>(A_all.size());
            term_offset.push_back(static_cast<std::int64_t>(A_all.size()));
            term_n.push_back(static_cast<int>(sec.size));
            A_all.insert(A_all.end(), A.begin(), A.end());
        }
        if (!invert_dense_blocks(A_all, term_offset, term_n, inv_all)) {
            throw Error(kESingular, "population_multigrid: singular block");
        }
        L->d_term.upload(L->h_term);
        L->inv64.upload(inv_all);
        std::vector<float> inv_f(inv_all.begin(), inv_all.end());
        L->inv32.upload(inv_f);
        if (opt.smoother == 3) {
            L->d_dense.upload(L->h_dense);
            L->dense64.upload(dense_all);
            L->dense32.upload(std::vector<float>(dense_all.begin(), dense_all.end()));
        }

        if (!next_totals.empty()) {
            // parent voxel of every fine voxel (multigrid.hpp:56-65)
            std::vector<int> parent;
            std::vector<double> log_children;
            parent_map(model.dim, dims, cdims, parent, log_children);
            L->parent.upload(parent);
            L->log_children.upload(log_children);
            if (opt.smoother == 3) {
                build_aggregates(*L, parent, static_cast<int>(log_children.size()));
            }
        } else if (opt.smoother == 3) {
            L->agg_ptr.assign(1, 0);
        }
        levels.push_back(std::move(L));
        totals = next_totals;
        box_of = next_box;
        for (int a = 0; a < 3; ++a) {
            dims[a] = cdims[a];
            spacing[a] = cspacing[a];
        }
        scale *= 2.0;
    }
    max_depth = static_cast<int>(levels.size());

    // work vectors in the preconditioner's precision, one column per right-hand side
    graph_exec_.assign(static_cast<std::size_t>(opt.batch) + 1, nullptr);
    graph_kernels_.assign(static_cast<std::size_t>(opt.batch) + 1, 0);
    for (std::size_t d = 0; d < levels.size(); ++d) {
        Level &L = *levels[d];
        // the FP32 batched cycle interleaves kRowBatch lanes whatever the batch width
        const std::size_t nb = static_cast<std::size_t>(
            opt.precision == 1 && opt.batch > 1 ? kRowBatch : opt.batch);
        const std::size_t nd = static_cast<std::size_t>(L.op.n) * nb;
        const std::size_t nc =
            d + 1 < levels.size() ? static_cast<std::size_t>(levels[d + 1]->op.n) * nb : 0;
        if (opt.precision == 0) {
            L.rhs64.resize(nd);
            L.x64.resize(nd);
            L.tmp64.resize(nd);
            L.r64.resize(nd);
            if (opt.coarse_cycles > 1 && nc) {
                L.acc64.resize(nc);
                L.crhs64.resize(nc);
            }
        } else {
            L.rhs32.resize(nd);
            L.x32.resize(nd);
            L.tmp32.resize(nd);
            L.r32.resize(nd);
            if (opt.coarse_cycles > 1 && nc) {
                L.acc32.resize(nc);
                L.crhs32.resize(nc);
            }
        }
    }
    if (opt.cycle_type == 1) {
        for (std::size_t d = 0; d + 2 < levels.size(); ++d) {
            Level &L = *levels[d];
            const std::size_t nc = static_cast<std::size_t>(levels[d + 1]->op.n);
            for (DeviceArray<double> *v : {&L.kg, &L.kv1, &L.kw1, &L.kv2, &L.kw2, &L.kr, &L.ke}) {
                v->resize(nc);
            }
            L.kdots.resize(8);
            L.kcoef.resize(4);
            L.kpartials.resize(kDotBlocks);
        }
    }
    build_transfers();
    if (opt.smoother == 2) {
        if (opt.precision == 0) {
            ilu_pivots<double>();
        } else {
            ilu_pivots<float>();
        }
    }
}

// Red-black ILU(0) pivots of every level: the diagonal (shift + exit) into a work vector, then
// P1 = D1 - diag(A10 D0^-1 A01) on the second colour. The diffusion-only level operator is
// bipartite in the checkerboard colour of the state (each jump moves one molecule to a
// neighbouring voxel, flipping the parity), so the elimination touches nothing but these pivots.
template <typename T>
void Multigrid::ilu_pivots() {
    for (auto &Lp : levels) {
        Level &L = *Lp;
        const std::size_t nd = static_cast<std::size_t>(L.op.n);
        DeviceArray<T> &piv = [&]() -> DeviceArray<T> & {
            if constexpr (std::is_same_v<T, double>) {
                return L.piv64;
            } else {
                return L.piv32;
            }
        }();
        piv.resize(nd);
        RowParams<T> p = L.op.params<T>();
        p.shift = static_cast<T>(shift);
        T *diag = buf<T>(L, 2);
        p.y = diag;
        L.op.run<T>(kDiagonal, p, nullptr);
        // first-colour rows keep their diagonal; second-colour rows get the modified pivot
        check_cuda(cudaMemcpyAsync(piv.get(), diag, nd * sizeof(T), cudaMemcpyDeviceToDevice, nullptr),
                   "pivot copy");
        p.aux = diag;
        p.y = piv.get();
        L.op.run<T>(kIluPivot, p, nullptr);
    }
    check_cuda(cudaStreamSynchronize(nullptr), "ILU(0) pivots");
}

template <typename T>
void Multigrid::ilu_sweep(Level &L, RowParams<T> p, T *x, const T *rhs, T *work,
                          cudaStream_t stream) {
    p.x = x;
    p.y = x;
    p.b = rhs;
    p.aux = work;
    if constexpr (std::is_same_v<T, double>) {
        p.piv = L.piv64.get();
    } else {
        p.piv = L.piv32.get();
    }
    L.op.run<T>(kIluFirst, p, stream);
    L.op.run<T>(kIluSecond, p, stream);
    L.op.run<T>(kIluThird, p, stream);
}

// The blocks of the aggregate-block smoother on one level (population_multigrid::build_blocks,
// markovkit/rdme/multigrid.hpp:266-299): for each coarse voxel a, the states of the non-terminal
// sectors grouped by their molecules outside a's fine voxels; groups of one state are skipped.
// Per block: its states (ascending), the rows of A = shift I - Q of those states and the dense
// inverse of A restricted to them (the reference factors the same matrix, multigrid.hpp:247-264).
void Multigrid::build_aggregates(Level &L, const std::vector<int> &parent, int coarse_voxels) {
    const OperatorLevel &op = L.op;
    const int V = op.V, S = op.S;
    const BinomTable B = op.binom->host_view();
    auto st = std::make_unique<RowState<kMaxSpecies, 64>>();
    // key: per species the count inside the coarse voxel, then the outside molecules
    std::vector<std::map<std::vector<int>, std::vector<std::int64_t>>> groups(
        static_cast<std::size_t>(coarse_voxels));
    for (const SectorDesc &sec : op.sectors) {
        if (sec.coarse < 0) {
            continue;
        }
        for (std::int64_t local = 0; local < sec.size; ++local) {
            load_state<kMaxSpecies, 64>(B, sec, S, V, local, *st);
            std::vector<int> seen;
            for (int s = 0; s < S; ++s) {
                for (int q = 0; q < sec.total[s]; ++q) {
                    const int a = parent[V - 1 - st->u[s][q]];
                    if (std::find(seen.begin(), seen.end(), a) != seen.end()) {
                        continue;
                    }
                    seen.push_back(a);
                    std::vector<int> key;
                    for (int s2 = 0; s2 < S; ++s2) {
                        int inside = 0;
                        for (int q2 = 0; q2 < sec.total[s2]; ++q2) {
                            inside += parent[V - 1 - st->u[s2][q2]] == a ? 1 : 0;
                        }
                        key.push_back(inside);
                        for (int q2 = 0; q2 < sec.total[s2]; ++q2) {
                            if (parent[V - 1 - st->u[s2][q2]] != a) {
                                key.push_back(st->u[s2][q2]);
                            }
                        }
                        key.push_back(-1);
                    }
                    groups[a][key].push_back(sec.begin + local);
                }
            }
        }
    }
    std::vector<AggBlock> blocks;
    std::vector<int> states, row_col;
    std::vector<std::int64_t> row_ptr{0};
    std::vector<double> row_val, inv_all, A, inv;
    L.agg_ptr.assign(1, 0);
    for (int a = 0; a < coarse_voxels; ++a) {
        for (auto &[key, members] : groups[a]) {
            if (members.size() < 2) {
                continue;
            }
            const int n = static_cast<int>(members.size());
            AggBlock blk;
            blk.state0 = static_cast<std::int64_t>(states.size());
            blk.inv0 = static_cast<std::int64_t>(inv_all.size());
            blk.n = n;
            A.assign(static_cast<std::size_t>(n) * n, 0.0);
            for (int k = 0; k < n; ++k) {
                const std::int64_t i = members[k];
                const int slot = [&] {
                    int q = 0;
                    while (q + 1 < static_cast<int>(op.sectors.size()) && op.sectors[q + 1].begin <= i) {
                        ++q;
                    }
                    return q;
                }();
                const SectorDesc &sec = op.sectors[slot];
                load_state<kMaxSpecies, 64>(B, sec, S, V, i - sec.begin, *st);
                double exit = 0.0, leak = 0.0;
                std::vector<std::pair<std::int64_t, double>> in;
                visit_row<double, kMaxSpecies, 64>(B, op.sectors.data(), sec, op.t64.host, i - sec.begin, *st,
                                                   true, 0, 1, exit, leak,
                                                   [&](std::int64_t j, double rate, double) { in.emplace_back(j, rate); });
                A[static_cast<std::size_t>(k) * n + k] += shift + exit;
                row_col.push_back(static_cast<int>(i));
                row_val.push_back(shift + exit);
                for (const auto &[j, rate] : in) {
                    row_col.push_back(static_cast<int>(j));
                    row_val.push_back(-rate);
                    const auto it = std::lower_bound(members.begin(), members.end(), j);
                    if (it != members.end() && *it == j) {
                        A[static_cast<std::size_t>(k) * n + (it - members.begin())] -= rate;
                    }
                }
                row_ptr.push_back(static_cast<std::int64_t>(row_col.size()));
                states.push_back(static_cast<int>(i));
            }
            if (!invert_dense(A, n, inv)) {
                throw Error(kESingular, "population_multigrid: singular block");
            }
            inv_all.insert(inv_all.end(), inv.begin(), inv.end());
            blocks.push_back(blk);
        }
        L.agg_ptr.push_back(static_cast<int>(blocks.size()));
    }
    L.agg_blocks.upload(blocks);
    L.agg_states.upload(states);
    L.agg_row_ptr.upload(row_ptr);
    L.agg_row_col.upload(row_col);
    if (opt.precision == 0) {
        L.agg_val64.upload(row_val);
        L.agg_inv64.upload(inv_all);
        L.agg_r64.resize(states.size());
        L.agg_e64.resize(states.size());
    } else {
        L.agg_val32.upload(std::vector<float>(row_val.begin(), row_val.end()));
        L.agg_inv32.upload(std::vector<float>(inv_all.begin(), inv_all.end()));
        L.agg_r32.resize(states.size());
        L.agg_e32.resize(states.size());
    }
}

// `sweeps` sweeps of the aggregate-block smoother on (rhs, x) (population_multigrid::smooth,
// markovkit/rdme/multigrid.hpp:319-341): block Gauss-Seidel over the coarse voxels in order
// (backwards when reverse), the blocks of one coarse voxel solved from the same residual; the
// terminal sectors take weighted Jacobi sweeps on their dense blocks (multigrid.hpp:309-317)
template <typename T>
void Multigrid::aggregate_smooth(Level &L, const T *rhs, T *x, T *scratch, int sweeps, bool reverse,
                                 bool from_zero, cudaStream_t stream) {
    const T *dense;
    AggView<T> v;
    v.blocks = L.agg_blocks.get();
    v.states = L.agg_states.get();
    v.row_ptr = L.agg_row_ptr.get();
    v.row_col = L.agg_row_col.get();
    if constexpr (std::is_same_v<T, double>) {
        dense = L.dense64.get();
        v.row_val = L.agg_val64.get();
        v.inv = L.agg_inv64.get();
        v.r = L.agg_r64.get();
        v.e = L.agg_e64.get();
    } else {
        dense = L.dense32.get();
        v.row_val = L.agg_val32.get();
        v.inv = L.agg_inv32.get();
        v.r = L.agg_r32.get();
        v.e = L.agg_e32.get();
    }
    check_cuda(launch_dense_jacobi<T>(L.d_dense.get(), static_cast<int>(L.h_dense.size()), dense, rhs, x,
                                      scratch, static_cast<T>(opt.jacobi_weight), sweeps, from_zero, stream),
               "dense Jacobi");
    const int aggregates = static_cast<int>(L.agg_ptr.size()) - 1;
    for (int sweep = 0; sweep < sweeps; ++sweep) {
        for (int step = 0; step < aggregates; ++step) {
            const int a = reverse ? aggregates - 1 - step : step;
            const int b0 = L.agg_ptr[a], b1 = L.agg_ptr[a + 1];
            if (b1 <= b0) {
                continue;
            }
            check_cuda(launch_aggregate_solve<T>(v, b0, b1, rhs, x, stream), "aggregate solve");
            check_cuda(launch_aggregate_update<T>(v, b0, b1, x, stream), "aggregate update");
        }
    }
}

int Multigrid::levels_of_sector(int k) const {
    int count = 0;
    for (const auto &L : levels) {
        if (std::find(L->box_sector.begin(), L->box_sector.end(), k) != L->box_sector.end()) {
            ++count;
        }
    }
    return count;
}

template <typename T>
T *Multigrid::buf(Level &L, int which, void *const *carve_level) {
    if (carve_level) {
        return static_cast<T *>(carve_level[which]);
    }
    if constexpr (std::is_same_v<T, double>) {
        switch (which) {
        case 0:
            return L.rhs64.get();
        case 1:
            return L.x64.get();
        case 2:
            return L.tmp64.get();
        case 3:
            return L.r64.get();
        case 4:
            return L.acc64.get();
        default:
            return L.crhs64.get();
        }
    } else {
        switch (which) {
        case 0:
            return L.rhs32.get();
        case 1:
            return L.x32.get();
        case 2:
            return L.tmp32.get();
        case 3:
            return L.r32.get();
        case 4:
            return L.acc32.get();
        default:
            return L.crhs32.get();
        }
    }
}

// one cycle of every sector at depth d from a zero initial guess
// (markovkit/rdme/multigrid.hpp:201-228); returns the buffer holding x
template <typename T>
T *Multigrid::cycle(int d, cudaStream_t stream, void *const *carve) {
    Level &L = *levels[d];
    void *const *cl = carve ? carve + 6 * d : nullptr;       // this level's caller vectors
    void *const *cc = carve ? carve + 6 * (d + 1) : nullptr; // the next level's
    const T *rhs = buf<T>(L, 0, cl);
    T *x = buf<T>(L, 1, cl);
    T *tmp = buf<T>(L, 2, cl);
    T *r = buf<T>(L, 3, cl);
    // nb_ columns: column c of every level vector at c * nd, except in the FP32 batched cycle,
    // whose kernels interleave kRowBatch lanes (entry (i, c) at i * kRowBatch + c)
    const std::int64_t nd = L.op.n;
    const int nb = nb_;
    const bool inter = std::is_same_v<T, float> && nb > 1;
    const int lanes = inter ? kRowBatch : nb;
    const std::int64_t ndb = nd * lanes;
    RowParams<T> p = L.op.params<T>();
    p.shift = static_cast<T>(shift);
    p.omega = static_cast<T>(opt.jacobi_weight);
    p.nb = nb;
    p.ldv = nd;

    if (opt.smoother == 0) {
        if (L.pre > 0) {
            p.b = rhs;
            p.y = x;
            L.op.run<T>(kJacobiZero, p, stream);
            for (int k = 1; k < L.pre; ++k) {
                p.x = x;
                p.b = rhs;
                p.y = tmp;
                L.op.run<T>(kJacobi, p, stream);
                std::swap(x, tmp);
            }
        } else {
            check_cuda(cudaMemsetAsync(x, 0, ndb * sizeof(T), stream), "memset");
        }
    } else if (opt.smoother == 1) {
        check_cuda(cudaMemsetAsync(x, 0, ndb * sizeof(T), stream), "memset");
        for (int k = 0; k < L.pre; ++k) {
            for (int q = 0; q < L.n_classes; ++q) {
                for (int c = 0; c < 2; ++c) {
                    p.b = rhs;
                    p.y = x;
                    p.colour = c;
                    p.sector_class = full_ ? q : -1;
                    L.op.run<T>(kGaussSeidel, p, stream);
                }
            }
        }
        p.sector_class = -1;
    } else if (opt.smoother == 2) {
        check_cuda(cudaMemsetAsync(x, 0, ndb * sizeof(T), stream), "memset");
        for (int k = 0; k < L.pre; ++k) {
            ilu_sweep<T>(L, p, x, rhs, tmp, stream);
        }
    } else {
        check_cuda(cudaMemsetAsync(x, 0, ndb * sizeof(T), stream), "memset");
        aggregate_smooth<T>(L, rhs, x, tmp, L.pre, false, true, stream);
    }

    // r = b - A x on every row; the coarse right-hand side is its restriction, summed in a
    // fixed order (terminal sectors keep r for their dense solve)
    Level *C = d + 1 < max_depth ? levels[d + 1].get() : nullptr;
    p.x = x;
    p.b = rhs;
    p.y = r;
    L.op.run<T>(kResidual, p, stream);
    if (C) {
        check_cuda(launch_restrict<T>(L.child_begin.get(), L.children.get(), C->op.n, r, nd,
                                      buf<T>(*C, 0, cc), C->op.n, nb, inter, stream),
                   "restrict");
    }
    if (!L.h_term.empty()) {
        const T *inv;
        if constexpr (std::is_same_v<T, double>) {
            inv = L.inv64.get();
        } else {
            inv = L.inv32.get();
        }
        int max_n = 0;
        for (const TerminalBlock &tb : L.h_term) {
            max_n = std::max(max_n, tb.n);
        }
        for (int c = 0; c < nb; ++c) {
            const std::int64_t off = inter ? c : c * nd;
            check_cuda(launch_terminal<T>(L.d_term.get(), static_cast<int>(L.h_term.size()),
                                          max_n, inv, r + off, x + off, inter ? lanes : 1, stream),
                       "terminal solve");
        }
    }
    if (C) {
        T *cx = nullptr;
        if constexpr (std::is_same_v<T, double>) {
            if (opt.cycle_type == 1 && d + 2 < max_depth) {
                cx = kcycle_coarse(d, stream);
            }
        }
        if (cx) {
            // the K-cycle's correction
        } else if (opt.coarse_cycles <= 1) {
            cx = cycle<T>(d + 1, stream, carve);
        } else {
            T *acc = buf<T>(L, 4, cl), *crhs = buf<T>(L, 5, cl);
            const std::size_t bytes = C->op.n * lanes * sizeof(T);
            check_cuda(cudaMemcpyAsync(crhs, buf<T>(*C, 0, cc), bytes, cudaMemcpyDeviceToDevice, stream),
                       "copy");
            T *e = cycle<T>(d + 1, stream, carve);
            check_cuda(cudaMemcpyAsync(acc, e, bytes, cudaMemcpyDeviceToDevice, stream), "copy");
            for (int c = 1; c < opt.coarse_cycles; ++c) {
                RowParams<T> pc = C->op.params<T>();
                pc.shift = static_cast<T>(shift);
                pc.x = acc;
                pc.b = crhs;
                pc.y = buf<T>(*C, 0, cc);
                pc.nb = nb;
                pc.ldv = C->op.n;
                C->op.run<T>(kResidual, pc, stream);
                e = cycle<T>(d + 1, stream, carve);
                axpy_t<T>(T(1), e, acc, C->op.n * lanes, stream);
            }
            cx = acc;
        }
        check_cuda(launch_prolong<T>(L.coarse_of.get(), weights<T>(L), nd, cx, C->op.n, x, nd, nb,
                                     inter, true, stream),
                   "prolong");
    }

    if (opt.smoother == 0) {
        for (int k = 0; k < L.post; ++k) {
            p.x = x;
            p.b = rhs;
            p.y = tmp;
            L.op.run<T>(kJacobi, p, stream);
            std::swap(x, tmp);
        }
    } else if (opt.smoother == 1) {
        for (int k = 0; k < L.post; ++k) {
            for (int q = L.n_classes - 1; q >= 0; --q) {
                for (int c = 1; c >= 0; --c) {
                    p.b = rhs;
                    p.y = x;
                    p.colour = c;
                    p.sector_class = full_ ? q : -1;
                    L.op.run<T>(kGaussSeidel, p, stream);
                }
            }
        }
        p.sector_class = -1;
    } else if (opt.smoother == 2) {
        for (int k = 0; k < L.post; ++k) {
            ilu_sweep<T>(L, p, x, rhs, tmp, stream);
        }
    } else {
        aggregate_smooth<T>(L, rhs, x, tmp, L.post, true, false, stream);
    }
    // keep the result in x's own buffer so the caller's view of the level stays fixed
    if (x != buf<T>(L, 1, cl)) {
        check_cuda(cudaMemcpyAsync(buf<T>(L, 1, cl), x, ndb * sizeof(T), cudaMemcpyDeviceToDevice,
                                   stream),
                   "copy");
    }
    return buf<T>(L, 1, cl);
}

namespace {

// The K-cycle's step coefficients from its dot products, on the device so that the cycle stays
// one captured graph (the reference's early returns become zero coefficients):
//   dots: 0 g.g, 1 w1.w1, 2 w1.g, 3 r.r, 4 w2.w1, 5 w2.w2, 6 w2.r
//   coef: 0 a1, 1 beta, 2 a2, 3 whether the second step is taken
__global__ void kcycle_coef_kernel(int phase, const double *dots, double *coef) {
    const bool first = dots[0] > 0.0 && dots[1] > 0.0;
    if (phase == 0) {
        coef[0] = first ? dots[2] / dots[1] : 0.0;
        coef[1] = coef[2] = coef[3] = 0.0;
    } else if (phase == 1) {
        const bool second = first && !(dots[3] <= 0.0625 * dots[0]);
        coef[3] = second ? 1.0 : 0.0;
        coef[1] = second ? dots[4] / dots[1] : 0.0;
    } else {
        coef[2] = coef[3] != 0.0 && dots[5] > 0.0 ? dots[6] / dots[5] : 0.0;
    }
}

// y = sign * coef[k] * x (init) or y += sign * coef[k] * x
__global__ void kcycle_axpy_kernel(const double *coef, int k, double sign, const double *x,
                                   double *y, std::int64_t n, bool init) {
    const double a = sign * coef[k];
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        y[i] = init ? a * x[i] : y[i] + a * x[i];
    }
}

void kcycle_axpy(const double *coef, int k, double sign, const double *x, double *y,
                 std::int64_t n, bool init, cudaStream_t stream) {
    const auto blocks = static_cast<unsigned>(std::clamp<std::int64_t>((n + 255) / 256, 1, 148 * 8));
    count_launches(1);
    kcycle_axpy_kernel<<<blocks, 256, 0, stream>>>(coef, k, sign, x, y, n, init);
    check_cuda(cudaGetLastError(), "K-cycle update");
}

} // namespace

// The K-cycle coarse solve of the paper driver (rdme/cpp/rdme_full_multigrid.cpp:851-878, after
// Notay and Vassilevski, in nonsymmetric GCR form): on A_c e = g at depth d + 1, at most two
// minimal-residual steps, each preconditioned by one recursive coarse cycle; the second step is
// skipped when the first reduces ||g|| by the factor 0.25 (here: taken with coefficient zero).
double *Multigrid::kcycle_coarse(int d, cudaStream_t stream) {
    Level &L = *levels[d];
    Level &C = *levels[d + 1];
    const std::int64_t n = C.op.n;
    const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(double);
    double *g = buf<double>(C, 0, nullptr);
    double *dots = L.kdots.get(), *coef = L.kcoef.get(), *part = L.kpartials.get();
    auto apply_c = [&](const double *v, double *w) {
        RowParams<double> p = C.op.params<double>();
        p.shift = shift;
        p.x = v;
        p.y = w;
        C.op.run<double>(kApplyShifted, p, stream);
    };
    auto dot_into = [&](const double *a, const double *b, int k) {
        check_cuda(dot(a, b, n, part, dots + k, stream), "K-cycle dot");
    };
    auto copy = [&](double *dst, const double *src) {
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream), "copy");
    };
    copy(L.kg.get(), g);
    dot_into(L.kg.get(), L.kg.get(), 0);
    copy(L.kv1.get(), cycle<double>(d + 1, stream, nullptr));
    apply_c(L.kv1.get(), L.kw1.get());
    dot_into(L.kw1.get(), L.kw1.get(), 1);
    dot_into(L.kw1.get(), L.kg.get(), 2);
    count_launches(3);
    kcycle_coef_kernel<<<1, 1, 0, stream>>>(0, dots, coef);
    kcycle_axpy(coef, 0, 1.0, L.kv1.get(), L.ke.get(), n, true, stream);
    copy(L.kr.get(), L.kg.get());
    kcycle_axpy(coef, 0, -1.0, L.kw1.get(), L.kr.get(), n, false, stream);
    dot_into(L.kr.get(), L.kr.get(), 3);
    copy(g, L.kr.get());
    copy(L.kv2.get(), cycle<double>(d + 1, stream, nullptr));
    apply_c(L.kv2.get(), L.kw2.get());
    dot_into(L.kw2.get(), L.kw1.get(), 4);
    kcycle_coef_kernel<<<1, 1, 0, stream>>>(1, dots, coef);
    kcycle_axpy(coef, 1, -1.0, L.kv1.get(), L.kv2.get(), n, false, stream);
    kcycle_axpy(coef, 1, -1.0, L.kw1.get(), L.kw2.get(), n, false, stream);
    dot_into(L.kw2.get(), L.kw2.get(), 5);
    dot_into(L.kw2.get(), L.kr.get(), 6);
    kcycle_coef_kernel<<<1, 1, 0, stream>>>(2, dots, coef);
    check_cuda(cudaGetLastError(), "K-cycle coefficients");
    kcycle_axpy(coef, 2, 1.0, L.kv2.get(), L.ke.get(), n, false, stream);
    return L.ke.get();
}

void Multigrid::transfer(int d, int direction, const double *in, double *out,
                         cudaStream_t stream) {
    if (d < 0 || d + 1 >= max_depth) {
        throw Error(kEInval, "no coarser level below this depth");
    }
    Level &L = *levels[d];
    Level &C = *levels[d + 1];
    if (direction == 0) {
        check_cuda(launch_restrict<double>(L.child_begin.get(), L.children.get(), C.op.n, in, L.op.n,
                                           out, C.op.n, 1, false, stream),
                   "restrict");
    } else {
        check_cuda(launch_prolong<double>(L.coarse_of.get(), L.w64.get(), L.op.n, in, C.op.n, out,
                                          L.op.n, 1, false, false, stream),
                   "prolong");
    }
}

// Per fine state of each non-terminal level: its coarse state and prolongation weight (one
// kCoarseIndex pass), then the children lists of the coarse states (one stable sort).
void Multigrid::build_transfers() {
    for (int d = 0; d + 1 < max_depth; ++d) {
        Level &L = *levels[d];
        Level &C = *levels[d + 1];
        const auto nf = static_cast<std::size_t>(L.op.n);
        L.coarse_of.resize(nf);
        L.w64.resize(nf);
        L.children.resize(nf);
        L.child_begin.resize(static_cast<std::size_t>(C.op.n) + 1);
        RowParams<double> p = L.op.params<double>();
        p.tv.Vc = C.op.V;
        p.tv.parent = L.parent.get();
        p.tv.log_children = L.log_children.get();
        p.tv.lgf = lgf.get();
        p.tv.coarse_sectors = C.op.d_sectors.get();
        p.idx = L.coarse_of.get();
        p.wout = L.w64.get();
        L.op.run<double>(kCoarseIndex, p, nullptr);
        DeviceArray<unsigned char> scratch(children_scratch_bytes(L.op.n));
        check_cuda(build_children(L.coarse_of.get(), L.op.n, C.op.n, L.children.get(),
                                  L.child_begin.get(), scratch.get(), scratch.size(), nullptr),
                   "multigrid children lists");
        if (opt.precision == 1) {
            L.w32.resize(nf);
            check_cuda(convert<double, float>(L.w64.get(), L.w32.get(), L.op.n, nullptr), "convert");
        }
        check_cuda(cudaStreamSynchronize(nullptr), "multigrid transfers");
    }
}

template <typename T>
const T *Multigrid::weights(const Level &L) const {
    if constexpr (std::is_same_v<T, double>) {
        return L.w64.get();
    } else {
        return L.w32.get();
    }
}

void Multigrid::apply_system(int d, const double *x, double *y, cudaStream_t stream) {
    if (d < 0 || d >= max_depth) {
        throw Error(kEInval, "no such multigrid level");
    }
    Level &L = *levels[d];
    RowParams<double> p = L.op.params<double>();
    p.shift = shift;
    p.x = x;
    p.y = y;
    L.op.run<double>(kApplyShifted, p, stream);
}

void Multigrid::smooth(int d, const double *b, double *x, cudaStream_t stream) {
    if (d < 0 || d >= max_depth) {
        throw Error(kEInval, "no such multigrid level");
    }
    if (opt.precision != 0) {
        throw Error(kEInval, "smooth: FP64 preconditioners only");
    }
    Level &L = *levels[d];
    RowParams<double> p = L.op.params<double>();
    p.shift = shift;
    p.omega = opt.jacobi_weight;
    double *tmp = buf<double>(L, 2);
    const std::size_t bytes = static_cast<std::size_t>(L.op.n) * sizeof(double);
    if (opt.smoother == 0) {
        p.x = x;
        p.b = b;
        p.y = tmp;
        L.op.run<double>(kJacobi, p, stream);
        check_cuda(cudaMemcpyAsync(x, tmp, bytes, cudaMemcpyDeviceToDevice, stream), "copy");
    } else if (opt.smoother == 1) {
        for (int c = 0; c < 2; ++c) {
            p.b = b;
            p.y = x;
            p.colour = c;
            L.op.run<double>(kGaussSeidel, p, stream);
        }
    } else if (opt.smoother == 2) {
        ilu_sweep<double>(L, p, x, b, tmp, stream);
    } else {
        aggregate_smooth<double>(L, b, x, tmp, 1, false, false, stream);
    }
}

// The cycle works only on the hierarchy's own buffers, so it is captured once into a CUDA
// graph (about six launches per level) and replayed on the caller's stream.
void Multigrid::ensure_graph(int nb) {
    if (graph_exec_[nb]) {
        return;
    }
    cudaStream_t cap = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream");
    cudaGraph_t graph = nullptr;
    nb_ = nb;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        try {
            if (opt.precision == 0) {
                cycle<double>(0, cap);
            } else {
                cycle<float>(0, cap);
            }
        } catch (...) {
            nb_ = 1;
            cudaStreamEndCapture(cap, &graph);
            if (graph) {
                cudaGraphDestroy(graph);
            }
            cudaStreamDestroy(cap);
            throw;
        }
        e = cudaStreamEndCapture(cap, &graph);
    }
    nb_ = 1;
    cudaStreamDestroy(cap);
    check_cuda(e, "multigrid graph capture");
    std::size_t n_nodes = 0;
    cudaGraphGetNodes(graph, nullptr, &n_nodes);
    std::vector<cudaGraphNode_t> nodes(n_nodes);
    cudaGraphGetNodes(graph, nodes.data(), &n_nodes);
    std::uint64_t kernels = 0;
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        if (cudaGraphNodeGetType(node, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) {
            ++kernels;
        }
    }
    graph_kernels_[nb] = kernels;
    e = cudaGraphInstantiate(&graph_exec_[nb], graph, 0);
    cudaGraphDestroy(graph);
    check_cuda(e, "multigrid graph instantiate");
}

namespace {
constexpr std::size_t kCarveAlign = 256;
std::size_t carve_round(std::size_t bytes) { return (bytes + kCarveAlign - 1) / kCarveAlign * kCarveAlign; }
} // namespace

std::size_t Multigrid::scratch_bytes() const {
    const std::size_t w = opt.precision == 0 ? sizeof(double) : sizeof(float);
    std::size_t total = 0;
    for (std::size_t d = 0; d < levels.size(); ++d) {
        const auto nd = static_cast<std::size_t>(levels[d]->op.n);
        total += 4 * carve_round(nd * w); // rhs, x, tmp, r
        if (opt.coarse_cycles > 1 && d + 1 < levels.size()) {
            total += 2 * carve_round(static_cast<std::size_t>(levels[d + 1]->op.n) * w); // acc, crhs
        }
    }
    return total;
}

void Multigrid::apply_in(const double *b, double *x, void *scratch, std::size_t bytes,
                         cudaStream_t stream) {
    if (bytes < scratch_bytes() || (reinterpret_cast<std::uintptr_t>(scratch) % kCarveAlign) != 0) {
        throw Error(kEInval, "multigrid scratch too small or misaligned");
    }
    if (opt.cycle_type == 1) {
        throw Error(kEInval, "the K-cycle keeps its vectors in the hierarchy");
    }
    // the work vectors of this call only: six per level, carved from the caller's memory and
    // handed down the cycle (the hierarchy's own buffers and state stay untouched)
    const std::size_t w = opt.precision == 0 ? sizeof(double) : sizeof(float);
    auto *base = static_cast<unsigned char *>(scratch);
    std::vector<void *> carve(6 * levels.size() + 6, nullptr);
    std::size_t off = 0;
    for (std::size_t d = 0; d < levels.size(); ++d) {
        const std::size_t vec = carve_round(static_cast<std::size_t>(levels[d]->op.n) * w);
        for (int k = 0; k < 4; ++k) {
            carve[6 * d + k] = base + off;
            off += vec;
        }
        if (opt.coarse_cycles > 1 && d + 1 < levels.size()) {
            const std::size_t cvec = carve_round(static_cast<std::size_t>(levels[d + 1]->op.n) * w);
            carve[6 * d + 4] = base + off;
            off += cvec;
            carve[6 * d + 5] = base + off;
            off += cvec;
        }
    }
    Level &L0 = *levels[0];
    const auto n0 = static_cast<std::int64_t>(L0.op.n);
    if (opt.precision == 0) {
        check_cuda(cudaMemcpyAsync(buf<double>(L0, 0, carve.data()), b, n0 * sizeof(double),
                                   cudaMemcpyDeviceToDevice, stream),
                   "copy");
        double *out = cycle<double>(0, stream, carve.data());
        check_cuda(cudaMemcpyAsync(x, out, n0 * sizeof(double), cudaMemcpyDeviceToDevice, stream),
                   "copy");
    } else {
        check_cuda(convert<double, float>(b, buf<float>(L0, 0, carve.data()), n0, stream), "convert");
        float *out = cycle<float>(0, stream, carve.data());
        check_cuda(convert<float, double>(out, x, n0, stream), "convert");
    }
}

Multigrid::~Multigrid() {
    for (cudaGraphExec_t g : graph_exec_) {
        if (g) {
            cudaGraphExecDestroy(g);
        }
    }
}

namespace {

// y[i * kRowBatch + c] = float(x[c * ldx + i]) for c < nb, 0 for the other lanes
__global__ void pack_lanes_kernel(const double *x, std::int64_t ldx, int nb, float *y,
                                  std::int64_t n) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        float v[kRowBatch];
#pragma unroll
        for (int c = 0; c < kRowBatch; ++c) {
            v[c] = c < nb ? static_cast<float>(x[c * ldx + i]) : 0.0f;
        }
        *reinterpret_cast<float4 *>(y + i * kRowBatch) = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// y[c * ldy + i] = double(x[i * kRowBatch + c]) for c < nb
__global__ void unpack_lanes_kernel(const float *x, std::int64_t n, int nb, double *y,
                                    std::int64_t ldy) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        const float4 v = *reinterpret_cast<const float4 *>(x + i * kRowBatch);
        const float u[kRowBatch] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int c = 0; c < kRowBatch; ++c) {
            if (c < nb) {
                y[c * ldy + i] = static_cast<double>(u[c]);
            }
        }
    }
}

unsigned lane_blocks(std::int64_t n) {
    return static_cast<unsigned>(std::max<std::int64_t>(1, std::min<std::int64_t>((n + 255) / 256, 148 * 8)));
}

} // namespace

static_assert(kRowBatch == 4, "the interleaved FP32 batch moves four lanes as one float4");

cudaError_t Multigrid::pack_lanes(const double *x, std::int64_t ldx, int nb, float *y,
                                  std::int64_t n, cudaStream_t stream) {
    count_launches(1);
    pack_lanes_kernel<<<lane_blocks(n), 256, 0, stream>>>(x, ldx, nb, y, n);
    return cudaGetLastError();
}

cudaError_t Multigrid::unpack_lanes(const float *x, std::int64_t n, int nb, double *y,
                                    std::int64_t ldy, cudaStream_t stream) {
    count_launches(1);
    unpack_lanes_kernel<<<lane_blocks(n), 256, 0, stream>>>(x, n, nb, y, ldy);
    return cudaGetLastError();
}

void Multigrid::apply(const double *b, double *x, cudaStream_t stream) {
    apply_batch(b, n, x, n, 1, stream);
}

void Multigrid::apply_batch(const double *b, std::int64_t ldb, double *x, std::int64_t ldx, int nb,
                            cudaStream_t stream) {
    if (nb < 1 || nb > opt.batch) {
        throw Error(kEInval, "multigrid: batch wider than the hierarchy was built for");
    }
    Level &L0 = *levels[0];
    const std::int64_t n0 = L0.op.n;
    ensure_graph(nb);
    const bool inter = opt.precision == 1 && nb > 1;
    if (inter) {
        check_cuda(pack_lanes(b, ldb, nb, L0.rhs32.get(), n0, stream), "pack");
    }
    for (int c = 0; c < nb && !inter; ++c) {
        if (opt.precision == 0) {
            check_cuda(cudaMemcpyAsync(L0.rhs64.get() + c * n0, b + c * ldb, n0 * sizeof(double),
                                       cudaMemcpyDeviceToDevice, stream),
                       "copy");
        } else {
            check_cuda(convert<double, float>(b + c * ldb, L0.rhs32.get() + c * n0, n0, stream),
                       "convert");
        }
    }
    check_cuda(cudaGraphLaunch(graph_exec_[nb], stream), "multigrid graph launch");
    count_launches(graph_kernels_[nb]);
    if (inter) {
        check_cuda(unpack_lanes(L0.x32.get(), n0, nb, x, ldx, stream), "unpack");
    }
    for (int c = 0; c < nb && !inter; ++c) {
        if (opt.precision == 0) {
            check_cuda(cudaMemcpyAsync(x + c * ldx, L0.x64.get() + c * n0, n0 * sizeof(double),
                                       cudaMemcpyDeviceToDevice, stream),
                       "copy");
        } else {
            check_cuda(convert<float, double>(L0.x32.get() + c * n0, x + c * ldx, n0, stream),
                       "convert");
        }
    }
}

// ---------------------------------------------------------------------------------------
// (F)GMRES

Krylov::Krylov(std::int64_t n_, int m_, bool flexible_) : n(n_), m(m_), flexible(flexible_) {
    if (m < 1) {
        throw Error(kEInval, "restart must be positive");
    }
    ld = (n + 31) / 32 * 32;
    V.resize(static_cast<std::size_t>(ld) * (m + 1));
    if (flexible) {
        Z.resize(static_cast<std::size_t>(ld) * m);
    }
    w.resize(ld);
    r.resize(ld);
    t.resize(ld);
    skip.resize(1);
    partials.resize(static_cast<std::size_t>(kDotBlocks) * kMaxFusedBasis);
    const std::size_t H = static_cast<std::size_t>(m + 1) * m;
    small.resize(H + 6 * (m + 1) + 16);
    double *p = small.get();
    st.m = m;
    st.H = p;
    p += H;
    st.cs = p;
    p += m + 1;
    st.sn = p;
    p += m + 1;
    st.g = p;
    p += m + 1;
    st.y = p;
    p += m + 1;
    st.h1 = p;
    p += m + 1;
    st.h2 = p;
    p += m + 1;
    st.hn = p++;
    st.inv_hn = p++;
    st.beta = p++;
    st.report = p;
    // slot 0: true residuals; slots 1 and 2: the two Arnoldi steps in flight
    check_cuda(cudaMallocHost(reinterpret_cast<void **>(&report_host), 12 * sizeof(double)),
               "cudaMallocHost");
    for (auto &e : step_done) {
        check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    }
}

Krylov::~Krylov() {
    for (auto &e : step_done) {
        if (e) {
            cudaEventDestroy(e);
        }
    }
    if (report_host) {
        cudaFreeHost(report_host);
    }
}

namespace {

// out[k] = <V_k, w> for k < K, any K
void gs_dots(const Krylov &ws, int K, double *w, double *out, cudaStream_t stream) {
    for (int c0 = 0; c0 < K; c0 += kMaxFusedBasis) {
        const int kc = std::min(kMaxFusedBasis, K - c0);
        check_cuda(cgs_pass(0, ws.V.get() + c0 * ws.ld, ws.ld, kc, w, ws.n, nullptr,
                            ws.partials.get(), out + c0, stream),
                   "cgs");
    }
}

// w -= V coef; then out = V^T w (mode 1) or out[0] = <w, w> (mode 2)
void gs_update(const Krylov &ws, int mode, int K, double *w, const double *coef, double *out,
               cudaStream_t stream) {
    if (K <= kMaxFusedBasis) {
        check_cuda(cgs_pass(mode, ws.V.get(), ws.ld, K, w, ws.n, coef, ws.partials.get(), out,
                            stream),
                   "cgs");
        return;
    }
    for (int c0 = 0; c0 < K; c0 += kMaxFusedBasis) {
        const int kc = std::min(kMaxFusedBasis, K - c0);
        check_cuda(cgs_pass(3, ws.V.get() + c0 * ws.ld, ws.ld, kc, w, ws.n, coef + c0,
                            ws.partials.get(), nullptr, stream),
                   "cgs");
    }
    if (mode == 1) {
        gs_dots(ws, K, w, out, stream);
    } else {
        check_cuda(dot(w, w, ws.n, ws.partials.get(), out, stream), "dot");
    }
}

void read_report(const Krylov &ws, cudaStream_t stream) {
    check_cuda(cudaMemcpyAsync(ws.report_host, ws.st.report, 4 * sizeof(double),
                               cudaMemcpyDeviceToHost, stream),
               "report");
    check_cuda(cudaStreamSynchronize(stream), "sync");
}

} // namespace

SolverResult stationary(const Generator &A, double shift, Preconditioner &M, const double *b,
                        double *x, double tol, std::int64_t max_cycles, cudaStream_t stream) {
    SolverResult res;
    const std::int64_t n = A.op.n;
    if (M.n != n) {
        throw Error(kEInval, "preconditioner size does not match the system");
    }
    DeviceArray<double> r(static_cast<std::size_t>(n)), z(static_cast<std::size_t>(n));
    DeviceArray<double> partials(kDotBlocks), norm2(1);
    for (std::int64_t it = 0;; ++it) {
        A.apply<double>(kResidual, shift, x, b, r.get(), nullptr, stream);
        check_cuda(dot(r.get(), r.get(), n, partials.get(), norm2.get(), stream), "dot");
        double h = 0.0;
        check_cuda(cudaMemcpyAsync(&h, norm2.get(), sizeof h, cudaMemcpyDeviceToHost, stream), "norm");
        check_cuda(cudaStreamSynchronize(stream), "sync");
        res.residual = std::sqrt(h);
        res.iterations = it;
        if (!std::isfinite(res.residual)) {
            res.status = kENan;
            return res;
        }
        if (res.residual <= tol) {
            res.converged = 1;
            return res;
        }
        if (it >= max_cycles) {
            res.status = kENotConv;
            return res;
        }
        M.apply(r.get(), z.get(), stream);
        check_cuda(axpy(1.0, z.get(), x, n, stream), "update");
    }
}

SolverResult gmres(const Generator &A, double shift, Preconditioner *M, const double *b,
                   double *x, const GmresOptions &opt, Krylov &ws, cudaStream_t stream) {
    SolverResult res;
    const std::int64_t n = A.op.n;
    if (ws.n != n) {
        throw Error(kEInval, "workspace size does not match the system");
    }
    if (M && M->n != n) {
        throw Error(kEInval, "preconditioner size does not match the system");
    }
    const bool flexible = opt.flexible || (M && M->varies());
    if (flexible && !ws.flexible) {
        throw Error(kEInval, "flexible GMRES needs a flexible workspace");
    }
    const int m = std::min(ws.m, std::max(1, opt.restart));
    const double tol = opt.tolerance;

    auto true_residual = [&]() {
        A.apply<double>(kResidual, shift, x, b, ws.r.get(), nullptr, stream);
        check_cuda(dot(ws.r.get(), ws.r.get(), n, ws.partials.get(), ws.st.beta, stream), "dot");
        check_cuda(arnoldi_start(ws.st, stream), "arnoldi");
        read_report(ws, stream);
        return ws.report_host[0];
    };

    double beta = true_residual();
    res.residual = beta;
    if (!std::isfinite(beta)) {
        res.status = kENan;
        return res;
    }
    if (beta <= tol) {
        res.converged = 1;
        return res;
    }
    while (res.iterations < opt.max_iterations) {
        check_cuda(scale_copy(ws.r.get(), ws.st.beta, ws.V.get(), n, stream), "scale");
        int k = 0;
        bool nan = false;
        // one Arnoldi step on the stream; its residual estimate lands in pinned slot j % 2
        auto enqueue = [&](int j) {
            double *vj = ws.V.get() + j * ws.ld;
            double *z = vj;
            if (M) {
                z = flexible ? ws.Z.get() + j * ws.ld : ws.t.get();
                M->apply(vj, z, stream);
            }
            A.apply<double>(kApplyShifted, shift, z, nullptr, ws.w.get(), nullptr, stream);
            const int K = j + 1;
            if (K < kMaxFusedBasis) {
                // the second (re-orthogonalisation) pass only where the first lost too much
                check_cuda(cgs_dgks(ws.V.get(), ws.ld, K, ws.w.get(), ws.n, ws.partials.get(),
                                    ws.st.h1, ws.st.h2, ws.st.hn, ws.skip.get(), stream),
                           "cgs");
            } else {
                gs_dots(ws, K, ws.w.get(), ws.st.h1, stream);
                gs_update(ws, 1, K, ws.w.get(), ws.st.h1, ws.st.h2, stream);
                gs_update(ws, 2, K, ws.w.get(), ws.st.h2, ws.st.hn, stream);
            }
            check_cuda(arnoldi_column(ws.st, j, stream), "arnoldi");
            double *slot = ws.report_host + 4 * (1 + (j & 1));
            check_cuda(cudaMemcpyAsync(slot, ws.st.report, 4 * sizeof(double),
                                       cudaMemcpyDeviceToHost, stream),
                       "report");
            check_cuda(cudaEventRecord(ws.step_done[j & 1], stream), "event");
            if (j + 1 < m) {
                check_cuda(scale_copy(ws.w.get(), ws.st.inv_hn, ws.V.get() + (j + 1) * ws.ld, n,
                                      stream),
                           "scale");
            }
        };
        // Step j + 1 is enqueued before the host waits for step j's estimate, so the host's
        // launch work overlaps the device's. When step j converges, step j + 1 has run but is
        // not used: the solve below takes the first k = j + 1 columns, and step j + 1 touched
        // only H's column j + 1 and g[j + 1..j + 2].
        const std::int64_t base = res.iterations; // steps taken in earlier restart cycles
        int enqueued = 0;
        if (base + 1 <= opt.max_iterations) {
            enqueue(0);
            enqueued = 1;
        }
        for (int j = 0; j < m && j < enqueued; ++j) {
            if (j + 1 < m && base + j + 2 <= opt.max_iterations) {
                enqueue(j + 1);
                ++enqueued;
            }
            check_cuda(cudaEventSynchronize(ws.step_done[j & 1]), "sync");
            const double *rep = ws.report_host + 4 * (1 + (j & 1));
            ++res.iterations;
            k = j + 1;
            if (!std::isfinite(rep[0]) || !std::isfinite(rep[1])) {
                nan = true;
                break;
            }
            if (rep[0] <= tol || rep[2] != 0.0) {
                break;
            }
        }
        check_cuda(cudaStreamSynchronize(stream), "sync");
        if (nan) {
            res.status = kENan;
            res.residual = std::numeric_limits<double>::quiet_NaN();
            return res;
        }
        check_cuda(arnoldi_solve(ws.st, k, stream), "arnoldi");
        if (flexible && M) {
            check_cuda(multi_axpy(ws.Z.get(), ws.ld, k, ws.st.y, x, n, stream), "update");
        } else if (M) {
            check_cuda(multi_combine(ws.V.get(), ws.ld, k, ws.st.y, ws.t.get(), n, stream), "update");
            M->apply(ws.t.get(), ws.w.get(), stream);
            check_cuda(axpy(1.0, ws.w.get(), x, n, stream), "update");
        } else {
            check_cuda(multi_axpy(ws.V.get(), ws.ld, k, ws.st.y, x, n, stream), "update");
        }
        beta = true_residual();
        res.residual = beta;
        if (!std::isfinite(beta)) {
            res.status = kENan;
            return res;
        }
        if (beta <= tol) {
            res.converged = 1;
            return res;
        }
    }
    res.status = kENotConv;
    return res;
}

// ---------------------------------------------------------------------------------------
// FGMRES for several right-hand sides in lockstep

namespace {

std::size_t arnoldi_small_size(int m) {
    return static_cast<std::size_t>(m + 1) * m + 6 * static_cast<std::size_t>(m + 1) + 16;
}

ArnoldiState carve_arnoldi(double *p, int m) {
    ArnoldiState st;
    st.m = m;
    st.H = p;
    p += static_cast<std::size_t>(m + 1) * m;
    st.cs = p;
    p += m + 1;
    st.sn = p;
    p += m + 1;
    st.g = p;
    p += m + 1;
    st.y = p;
    p += m + 1;
    st.h1 = p;
    p += m + 1;
    st.h2 = p;
    p += m + 1;
    st.hn = p++;
    st.inv_hn = p++;
    st.beta = p++;
    st.report = p;
    return st;
}

} // namespace

KrylovBatch::KrylovBatch(std::int64_t n_, int m_, int nb_) : n(n_), m(m_), nb(nb_) {
    if (m < 1 || nb < 1) {
        throw Error(kEInval, "restart and batch must be positive");
    }
    ld = (n + 31) / 32 * 32;
    V.resize(static_cast<std::size_t>(ld) * nb * (m + 1));
    Z.resize(static_cast<std::size_t>(ld) * nb * m);
    w.resize(static_cast<std::size_t>(ld) * nb);
    r.resize(static_cast<std::size_t>(ld) * nb);
    partials.resize(static_cast<std::size_t>(kDotBlocks) * kMaxFusedBasis * nb);
    reports.resize(static_cast<std::size_t>(4) * nb);
    const std::size_t per = arnoldi_small_size(m);
    small_stride = static_cast<std::int64_t>(per);
    small.resize(per * nb);
    for (int c = 0; c < nb; ++c) {
        st.push_back(carve_arnoldi(small.get() + per * c, m));
    }
    check_cuda(cudaMallocHost(reinterpret_cast<void **>(&report_host), 8 * sizeof(double) * nb),
               "cudaMallocHost");
    for (auto &e : step_done) {
        check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    }
}

KrylovBatch::~KrylovBatch() {
    for (auto &e : step_done) {
        if (e) {
            cudaEventDestroy(e);
        }
    }
    if (report_host) {
        cudaFreeHost(report_host);
    }
}

std::vector<SolverResult> gmres_batch(const Generator &A, double shift, Multigrid &M,
                                      const double *b, double *x, int nb, const double *tol,
                                      const GmresOptions &opt, KrylovBatch &ws,
                                      cudaStream_t stream) {
    const std::int64_t n = A.op.n, ld = ws.ld;
    if (ws.n != n || M.n != n) {
        throw Error(kEInval, "workspace or preconditioner size does not match the system");
    }
    if (nb < 1 || nb > ws.nb || nb > M.opt.batch) {
        throw Error(kEInval, "batch wider than the workspace or the multigrid");
    }
    const int m = std::min(ws.m, std::max(1, opt.restart));
    std::vector<SolverResult> res(nb);
    std::vector<char> active(nb, 1);
    auto col = [&](const double *base, int c) { return base + c * ld; };
    // basis vector j of column c and its stride inside the column
    auto Vj = [&](int j, int c) { return ws.V.get() + (static_cast<std::int64_t>(j) * ws.nb + c) * ld; };
    auto Zj = [&](int j, int c) { return ws.Z.get() + (static_cast<std::int64_t>(j) * ws.nb + c) * ld; };
    const std::int64_t col_stride = static_cast<std::int64_t>(ws.nb) * ld;

    auto read_reports = [&]() {
        check_cuda(cudaStreamSynchronize(stream), "sync");
    };
    // r = b - A x for every column, beta_c = ||r_c||; returns false on a non-finite residual
    auto true_residuals = [&]() {
        A.apply<double>(kResidual, shift, x, b, ws.r.get(), nullptr, stream, nb, ld);
        for (int c = 0; c < nb; ++c) {
            check_cuda(dot(col(ws.r.get(), c), col(ws.r.get(), c), n, ws.partials.get(),
                           ws.st[c].beta, stream),
                       "dot");
            check_cuda(arnoldi_start(ws.st[c], stream), "arnoldi");
            check_cuda(cudaMemcpyAsync(ws.report_host + 4 * c, ws.st[c].report, 4 * sizeof(double),
                                       cudaMemcpyDeviceToHost, stream),
                       "report");
        }
        read_reports();
        for (int c = 0; c < nb; ++c) {
            if (!active[c]) {
                continue;
            }
            const double beta = ws.report_host[4 * c];
            res[c].residual = beta;
            if (!std::isfinite(beta)) {
                res[c].status = kENan;
                active[c] = 0;
            } else if (beta <= tol[c]) {
                res[c].converged = 1;
                active[c] = 0;
            } else if (res[c].iterations >= opt.max_iterations) {
                res[c].status = kENotConv;
                active[c] = 0;
            }
        }
    };

    true_residuals();
    while (std::count(active.begin(), active.end(), 1) > 0) {
        std::vector<int> k(nb, 0);
        std::vector<char> running(active);
        for (int c = 0; c < nb; ++c) {
            if (running[c]) {
                check_cuda(scale_copy(col(ws.r.get(), c), ws.st[c].beta, Vj(0, c), n, stream), "scale");
            }
        }
        // Step j of every column still running when it is enqueued; its estimates land in
        // pinned slot j % 2. Step j + 1 is enqueued before the host waits for step j, as in
        // the single-column solver: a column that converges at step j ignores step j + 1,
        // which touched only its H column j + 1, g[j + 1..] and basis vector j + 2.
        auto enqueue = [&](int j, const std::vector<char> &cols) {
            // one multigrid cycle and one operator apply serve every column of step j
            M.apply_batch(Vj(j, 0), ld, Zj(j, 0), ld, nb, stream);
            A.apply<double>(kApplyShifted, shift, Zj(j, 0), nullptr, ws.w.get(), nullptr, stream,
                            nb, ld);
            if (j + 1 <= kMaxFusedBasis && nb <= 32) {
                // every running column's Gram-Schmidt, Givens column and next basis vector in
                // one launch per pass, and one copy of their reports
                ColumnBatch cb;
                cb.V = ws.V.get();
                cb.vstride = col_stride;
                cb.w = ws.w.get();
                cb.col = ld;
                cb.st = ws.st[0];
                cb.small = ws.small_stride;
                cb.partials = ws.partials.get();
                cb.reports = ws.reports.get();
                cb.nb = nb;
                cb.n = n;
                for (int c = 0; c < nb; ++c) {
                    cb.mask |= cols[c] ? (1U << c) : 0U;
                }
                check_cuda(cgs_step_batch(cb, j, j + 1 < m, stream), "batched Gram-Schmidt");
                check_cuda(cudaMemcpyAsync(ws.report_host + 4 * nb * (j & 1), ws.reports.get(),
                                           4 * nb * sizeof(double), cudaMemcpyDeviceToHost, stream),
                           "report");
                check_cuda(cudaEventRecord(ws.step_done[j & 1], stream), "event");
                return;
            }
            for (int c = 0; c < nb; ++c) {
                if (!cols[c]) {
                    continue;
                }
                double *w = ws.w.get() + c * ld;
                const int K = j + 1;
                const double *Vc = Vj(0, c);
                for (int c0 = 0; c0 < K; c0 += kMaxFusedBasis) {
                    const int kc = std::min(kMaxFusedBasis, K - c0);
                    check_cuda(cgs_pass(0, Vc + c0 * col_stride, col_stride, kc, w, n, nullptr,
                                        ws.partials.get(), ws.st[c].h1 + c0, stream),
                               "cgs");
                }
                for (int pass = 1; pass <= 2; ++pass) {
                    const double *coef = pass == 1 ? ws.st[c].h1 : ws.st[c].h2;
                    double *out = pass == 1 ? ws.st[c].h2 : ws.st[c].hn;
                    if (K <= kMaxFusedBasis) {
                        check_cuda(cgs_pass(pass, Vc, col_stride, K, w, n, coef, ws.partials.get(),
                                            out, stream),
                                   "cgs");
                    } else {
                        for (int c0 = 0; c0 < K; c0 += kMaxFusedBasis) {
                            const int kc = std::min(kMaxFusedBasis, K - c0);
                            check_cuda(cgs_pass(3, Vc + c0 * col_stride, col_stride, kc, w, n,
                                                coef + c0, ws.partials.get(), nullptr, stream),
                                       "cgs");
                        }
                        if (pass == 1) {
                            for (int c0 = 0; c0 < K; c0 += kMaxFusedBasis) {
                                const int kc = std::min(kMaxFusedBasis, K - c0);
                                check_cuda(cgs_pass(0, Vc + c0 * col_stride, col_stride, kc, w, n,
                                                    nullptr, ws.partials.get(), out + c0, stream),
                                           "cgs");
                            }
                        } else {
                            check_cuda(dot(w, w, n, ws.partials.get(), out, stream), "dot");
                        }
                    }
                }
                check_cuda(arnoldi_column(ws.st[c], j, stream), "arnoldi");
                double *slot = ws.report_host + 4 * (nb * (j & 1) + c);
                check_cuda(cudaMemcpyAsync(slot, ws.st[c].report, 4 * sizeof(double),
                                           cudaMemcpyDeviceToHost, stream),
                           "report");
                if (j + 1 < m) {
                    check_cuda(scale_copy(w, ws.st[c].inv_hn, Vj(j + 1, c), n, stream), "scale");
                }
            }
            check_cuda(cudaEventRecord(ws.step_done[j & 1], stream), "event");
        };
        std::vector<int> steps_left(nb);
        for (int c = 0; c < nb; ++c) {
            steps_left[c] = static_cast<int>(
                std::min<std::int64_t>(m, std::max<std::int64_t>(0, opt.max_iterations - res[c].iterations)));
        }
        enqueue(0, running);
        for (int j = 0; j < m; ++j) {
            bool next = false;
            for (int c = 0; c < nb; ++c) {
                next = next || (running[c] && j + 1 < steps_left[c]);
            }
            if (next && j + 1 < m) {
                enqueue(j + 1, running);
            }
            check_cuda(cudaEventSynchronize(ws.step_done[j & 1]), "sync");
            bool any = false;
            for (int c = 0; c < nb; ++c) {
                if (!running[c]) {
                    continue;
                }
                const double *rep = ws.report_host + 4 * (nb * (j & 1) + c);
                ++res[c].iterations;
                k[c] = j + 1;
                if (!std::isfinite(rep[0]) || !std::isfinite(rep[1])) {
                    res[c].status = kENan;
                    active[c] = 0;
                    running[c] = 0;
                    continue;
                }
                if (rep[0] <= tol[c] || rep[2] != 0.0 || j + 1 >= steps_left[c]) {
                    running[c] = 0; // this cycle ends here for column c
                    continue;
                }
                any = true;
            }
            if (!any || !next) {
                break;
            }
        }
        check_cuda(cudaStreamSynchronize(stream), "sync");
        for (int c = 0; c < nb; ++c) {
            if (!active[c] || k[c] == 0) {
                continue;
            }
            check_cuda(arnoldi_solve(ws.st[c], k[c], stream), "arnoldi");
            check_cuda(multi_axpy(Zj(0, c), col_stride, k[c], ws.st[c].y, x + c * ld, n, stream),
                       "update");
        }
        true_residuals();
    }
    return res;
}

} // namespace mkb
