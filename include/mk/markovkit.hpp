// markovkit_b200 C++20 facade: MarkovKit's resolvent-path and Krylov-FSP API (names, argument
// meaning, exceptions) over the C ABI of include/markovkit_b200.h. Header-only; link
// libmarkovkit_b200.so. Vectors are host std::vectors, as in the reference; every call copies
// them to the device, runs the sm_100a kernels and copies back, synchronously (the reference's
// calls are synchronous too). Handles own device memory and free it on destruction.
//
// Reference interfaces mirrored (MarkovKit tree):
//   population_box / population_sector        markovkit/rdme/population_space.hpp:105-196
//   grid<D>, voxel_domain, local_reaction,
//   reaction_diffusion                         markovkit/rdme/reaction_diffusion.hpp:15-118
//   boundary, generator, shifted_generator     markovkit/generator.hpp:11-133
//   multigrid_options, sector_multigrid        markovkit/rdme/multigrid.hpp:125-134,364-408
//   num::gmres_options, num::solver_result,
//   num::gmres(A, [M], b, x, options),
//   num::jacobi_preconditioner,
//   num::ilu0_preconditioner                   call sites tests/test_rdme.cpp:238-249,
//                                              examples/rdme_multigrid_benchmark.cpp:82-115
//   generator::jumps(j), exit_rates()          markovkit/generator.hpp:22-59
//   reaction_network, box, krylov_fsp_options,
//   adaptive_fsp_options, fsp_solution,
//   solve_krylov_fsp, solve_adaptive_fsp       markovkit/reaction_network.hpp, fsp.hpp:26-254
// Differences: the voxel graph is a structured grid (grid<1..3>); a region for FSP is a box;
// krylov_dim <= 30; fsp_solution keeps the initial and final snapshots only.
#pragma once

#include "../markovkit_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <concepts>
#include <cstdint>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <optional>
#include <random>
#include <span>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace markovkit {

using real = double;
using idx = std::size_t;
template <typename T>
using vec = std::vector<T>;
template <typename T>
using array = std::vector<T>;
template <typename T>
using view = std::span<T>;
using state = std::vector<int>;

// the numerics library's names the reference's programs use through `num::`
namespace num {
using markovkit::real;
using markovkit::idx;
template <typename T>
using vec = std::vector<T>;
template <typename T>
using array = std::vector<T>;
template <typename T, std::size_t N>
using static_array = std::array<T, N>;

// a seeded uniform random bit generator, the numerics library's num::rng as MarkovKit's
// programs use it (tests/test_ssa.cpp:27): here it only seeds the device streams of
// gillespie and tau_leaping
class rng {
  public:
    using result_type = std::uint64_t;
    explicit rng(std::uint64_t seed = 0) : engine_(seed) {}
    static constexpr result_type min() { return std::mt19937_64::min(); }
    static constexpr result_type max() { return std::mt19937_64::max(); }
    result_type operator()() { return engine_(); }

  private:
    std::mt19937_64 engine_;
};
} // namespace num

namespace detail {

inline void check(int rc) {
    if (rc == MK_OK) {
        return;
    }
    const std::string msg = mk_last_error();
    switch (rc) {
    case MK_EINVAL:
        throw std::invalid_argument(msg);
    case MK_EOVERFLOW:
        throw std::overflow_error(msg);
    case MK_ENOMEM:
        throw std::bad_alloc();
    default:
        throw std::runtime_error(msg);
    }
}

// a device buffer of doubles for host-vector calls
class device_vector {
  public:
    device_vector() = default;
    explicit device_vector(std::size_t n) : n_(n) {
        void *p = nullptr;
        check(mk_device_alloc(n * sizeof(double), &p));
        p_.reset(static_cast<double *>(p));
    }
    [[nodiscard]] double *get() const { return p_.get(); }
    [[nodiscard]] std::size_t size() const { return n_; }
    void upload(const double *h) { check(mk_memcpy_h2d(p_.get(), h, n_ * sizeof(double), nullptr)); }
    void download(double *h) const {
        check(mk_memcpy_d2h(h, p_.get(), n_ * sizeof(double), nullptr));
        check(mk_stream_synchronize(nullptr));
    }

  private:
    struct freer {
        void operator()(double *p) const { mk_device_free(p); }
    };
    std::unique_ptr<double, freer> p_;
    std::size_t n_ = 0;
};

template <typename H, void (*Destroy)(H)>
struct handle_deleter {
    void operator()(H h) const {
        if (h) {
            Destroy(h);
        }
    }
};

} // namespace detail

// ---- spaces ------------------------------------------------------------------------------

class population_space {
  public:
    [[nodiscard]] idx size() const {
        int64_t n = 0;
        detail::check(mk_space_size(h_.get(), &n));
        return static_cast<idx>(n);
    }
    [[nodiscard]] idx n_voxels() const { return static_cast<idx>(voxels_); }
    [[nodiscard]] idx n_species() const { return limits_.size(); }
    [[nodiscard]] idx n_sectors() const {
        int64_t k = 0;
        detail::check(mk_space_n_sectors(h_.get(), &k));
        return static_cast<idx>(k);
    }
    [[nodiscard]] idx sector_begin(idx k) const {
        int64_t b = 0;
        detail::check(mk_space_sector_begin(h_.get(), static_cast<int64_t>(k), &b));
        return static_cast<idx>(b);
    }
    [[nodiscard]] idx sector_end(idx k) const {
        return k + 1 < n_sectors() ? sector_begin(k + 1) : size();
    }
    [[nodiscard]] array<int> sector_totals(idx k) const {
        array<int> t(n_species());
        detail::check(mk_space_sector_totals(h_.get(), static_cast<int64_t>(k), t.data()));
        return t;
    }
    [[nodiscard]] idx sector_of(idx i) const {
        int64_t k = 0;
        detail::check(mk_space_sector_of(h_.get(), static_cast<int64_t>(i), &k));
        return static_cast<idx>(k);
    }
    [[nodiscard]] std::optional<idx> find_sector(const array<int> &totals) const {
        int64_t k = -1;
        detail::check(mk_space_find_sector(h_.get(), totals.data(), &k));
        return k < 0 ? std::nullopt : std::optional<idx>(static_cast<idx>(k));
    }
    // find(x): the index of a voxel-major occupation vector, or nullopt
    [[nodiscard]] std::optional<idx> find(const state &x) const {
        if (x.size() != n_voxels() * n_species()) {
            return std::nullopt;
        }
        int64_t i = -1;
        detail::check(mk_space_find_host(h_.get(), x.data(), &i));
        return i < 0 ? std::nullopt : std::optional<idx>(static_cast<idx>(i));
    }
    [[nodiscard]] state operator[](idx i) const {
        state x(n_voxels() * n_species());
        detail::check(mk_space_state_host(h_.get(), static_cast<int64_t>(i), x.data()));
        return x;
    }
    [[nodiscard]] mk_space handle() const { return h_.get(); }
    [[nodiscard]] const array<int> &limits() const { return limits_; }

  protected:
    population_space(idx voxels, array<int> limits, bool box)
        : voxels_(static_cast<int64_t>(voxels)), limits_(std::move(limits)) {
        mk_space h = nullptr;
        detail::check(box ? mk_space_create_box(voxels_, static_cast<int>(limits_.size()),
                                                limits_.data(), &h)
                          : mk_space_create_sector(voxels_, static_cast<int>(limits_.size()),
                                                   limits_.data(), &h));
        h_ = std::shared_ptr<mk_space_s>(h, [](mk_space p) { mk_space_destroy(p); });
    }

  private:
    int64_t voxels_ = 0;
    array<int> limits_;
    std::shared_ptr<mk_space_s> h_;
};

// every sector 0 <= t_s <= max_totals[s]
class population_box : public population_space {
  public:
    population_box(idx voxels, array<int> max_totals)
        : population_space(voxels, std::move(max_totals), true) {}
};

// the states with totals[s] molecules of each species
class population_sector : public population_space {
  public:
    population_sector(idx voxels, array<int> totals)
        : population_space(voxels, std::move(totals), false) {}
};

// ---- models -------------------------------------------------------------------------------

// a jump out of a state (chain.hpp:33-36)
struct transition {
    state to;
    real rate;
};

// a model lists every jump out of a state with a positive rate (chain.hpp:38-42)
template <typename Model>
concept markov_model = requires(const Model &model, const state &x) {
    { model.transitions(x) } -> std::convertible_to<array<transition>>;
};

// a finite state space numbers its states 0, ..., size() - 1 (chain.hpp:44-50)
template <typename Space>
concept state_space = requires(const Space &space, const state &x, idx i) {
    { space.size() } -> std::convertible_to<idx>;
    { space[i] } -> std::convertible_to<const state &>;
    { space.find(x) } -> std::convertible_to<std::optional<idx>>;
};

// grid<D>(dims, spacing): a structured voxel grid (the reference's structured_grid_graph):
// vertex numbering with axis 0 fastest, closed boundary, neighbours axis by axis with the lower
// one first, edge weight = face area / h
template <int D>
struct grid {
    struct edge {
        idx to;
        real weight;
    };
    std::array<idx, D> dims;
    std::array<real, D> spacing;
    explicit grid(std::array<idx, D> d) : dims(d) { spacing.fill(1.0); }
    grid(std::array<idx, D> d, std::array<real, D> h) : dims(d), spacing(h) {}
    [[nodiscard]] idx n_vertices() const {
        idx n = 1;
        for (idx d : dims) {
            n *= d;
        }
        return n;
    }
    [[nodiscard]] real cell_volume() const {
        real v = 1.0;
        for (real h : spacing) {
            v *= h;
        }
        return v;
    }
    [[nodiscard]] array<edge> neighbors(idx v) const {
        array<edge> out;
        idx stride = 1, rem = v;
        for (int a = 0; a < D; ++a) {
            const idx c = rem % dims[a];
            rem /= dims[a];
            real face = 1.0;
            for (int b = 0; b < D; ++b) {
                if (b != a) {
                    face *= spacing[b];
                }
            }
            const real w = face / spacing[a];
            if (c > 0) {
                out.push_back({v - stride, w});
            }
            if (c + 1 < dims[a]) {
                out.push_back({v + stride, w});
            }
            stride *= dims[a];
        }
        return out;
    }
};

namespace num {

// an explicit undirected weighted graph (the numerics library's graph<W, I>):
// add_edge(a, b, w) adds a -> b and b -> a
template <typename W = double, typename I = idx>
class graph {
  public:
    struct edge {
        I to;
        W weight;
    };
    explicit graph(I n = 0) : adj_(n) {}
    void add_edge(I a, I b, W weight) {
        adj_.at(a).push_back({b, weight});
        adj_.at(b).push_back({a, weight});
    }
    [[nodiscard]] I n_vertices() const { return static_cast<I>(adj_.size()); }
    [[nodiscard]] const array<edge> &neighbors(I v) const { return adj_.at(v); }

  private:
    array<array<edge>> adj_;
};

} // namespace num

// voxel_domain(graph, [volumes,] diffusivities) (reaction_diffusion.hpp:23-56): a grid's
// volumes are its cell volume
template <typename Graph>
struct voxel_domain {
    Graph graph;
    vec<real> diffusivities;
    vec<real> volumes;
    voxel_domain(Graph g, vec<real> diff)
        requires requires(const Graph &x) { x.cell_volume(); }
        : graph(std::move(g)), diffusivities(std::move(diff)),
          volumes(graph.n_vertices(), graph.cell_volume()) {}
    voxel_domain(Graph g, vec<real> vols, vec<real> diff)
        : graph(std::move(g)), diffusivities(std::move(diff)), volumes(std::move(vols)) {
        if (volumes.size() != static_cast<idx>(graph.n_vertices())) {
            throw std::invalid_argument("voxel_domain: one volume per voxel");
        }
    }
    [[nodiscard]] idx n_voxels() const { return static_cast<idx>(graph.n_vertices()); }
    [[nodiscard]] idx n_species() const { return diffusivities.size(); }
    // the rate at which one molecule of a species hops along an edge out of a voxel
    template <typename Edge>
    [[nodiscard]] real jump_rate(idx species, idx from, const Edge &edge) const {
        return diffusivities[species] * static_cast<real>(edge.weight) / volumes[from];
    }
};

// a reaction inside one voxel: change vector and rate(counts, volume)
struct local_reaction {
    array<int> change;
    std::function<real(view<const int>, real)> rate;
};

template <typename Graph>
struct reaction_diffusion {
    voxel_domain<Graph> domain;
    array<local_reaction> reactions;
    [[nodiscard]] idx n_voxels() const { return domain.n_voxels(); }
    [[nodiscard]] idx n_species() const { return domain.n_species(); }
    [[nodiscard]] idx index(idx voxel, idx species) const { return voxel * n_species() + species; }
    // every jump out of x (reaction_diffusion.hpp:82-118): diffusion by voxel, edge and species,
    // then local reactions by voxel; a host-side enumeration for callers (the device kernels
    // visit the same jumps)
    [[nodiscard]] array<transition> transitions(const state &x) const {
        array<transition> result;
        const idx S = n_species();
        for (idx v = 0; v < n_voxels(); ++v) {
            for (const auto &edge : domain.graph.neighbors(v)) {
                for (idx s = 0; s < S; ++s) {
                    const int n = x[index(v, s)];
                    if (n == 0) {
                        continue;
                    }
                    state y = x;
                    --y[index(v, s)];
                    ++y[index(static_cast<idx>(edge.to), s)];
                    result.push_back({std::move(y), n * domain.jump_rate(s, v, edge)});
                }
            }
        }
        for (idx v = 0; v < n_voxels(); ++v) {
            const view<const int> counts(x.data() + index(v, 0), S);
            for (const local_reaction &r : reactions) {
                const real rate = r.rate(counts, domain.volumes[v]);
                if (!(rate > 0.0)) {
                    continue;
                }
                state y = x;
                bool valid = true;
                for (idx s = 0; s < S; ++s) {
                    y[index(v, s)] += r.change[s];
                    valid = valid && y[index(v, s)] >= 0;
                }
                if (valid) {
                    result.push_back({std::move(y), rate});
                }
            }
        }
        return result;
    }
};

namespace detail {

template <typename G>
struct is_grid : std::false_type {};
template <int D>
struct is_grid<grid<D>> : std::true_type {};

// the model handle of a reaction-diffusion model with its local rates tabulated over the
// count tuples a space allows (n_s <= limits[s]), one table per distinct voxel volume
template <typename Graph>
std::shared_ptr<mk_model_s> make_model(const reaction_diffusion<Graph> &m, const array<int> &limits) {
    const auto &dom = m.domain;
    const int S = static_cast<int>(m.n_species());
    mk_model h = nullptr;
    if constexpr (is_grid<Graph>::value) {
        constexpr int D = static_cast<int>(std::tuple_size_v<decltype(dom.graph.dims)>);
        std::array<int64_t, 3> dims{1, 1, 1};
        std::array<double, 3> spacing{1.0, 1.0, 1.0};
        for (int a = 0; a < D; ++a) {
            dims[a] = static_cast<int64_t>(dom.graph.dims[a]);
            spacing[a] = dom.graph.spacing[a];
        }
        check(mk_model_create_grid(D, dims.data(), spacing.data(), S, dom.diffusivities.data(), &h));
    } else {
        const idx V = dom.n_voxels();
        std::vector<int64_t> ptr{0}, nbr;
        std::vector<double> w;
        for (idx v = 0; v < V; ++v) {
            for (const auto &e : dom.graph.neighbors(static_cast<decltype(dom.graph.n_vertices())>(v))) {
                nbr.push_back(static_cast<int64_t>(e.to));
                w.push_back(static_cast<double>(e.weight));
            }
            ptr.push_back(static_cast<int64_t>(nbr.size()));
        }
        check(mk_model_create_graph(static_cast<int64_t>(V), ptr.data(), nbr.data(), w.data(),
                                    dom.volumes.data(), S, dom.diffusivities.data(), &h));
    }
    std::shared_ptr<mk_model_s> model(h, [](mk_model p) { mk_model_destroy(p); });
    if (!m.reactions.empty()) {
        if (static_cast<int>(limits.size()) != S) {
            throw std::invalid_argument("the space and the model have different species counts");
        }
        int ntuple = 1;
        for (int t : limits) {
            ntuple *= t + 1;
        }
        // volume classes: the distinct voxel volumes, in order of first appearance
        std::vector<double> classes;
        std::vector<int> vclass(dom.n_voxels());
        for (idx v = 0; v < dom.n_voxels(); ++v) {
            const auto it = std::find(classes.begin(), classes.end(), dom.volumes[v]);
            vclass[v] = static_cast<int>(it - classes.begin());
            if (it == classes.end()) {
                classes.push_back(dom.volumes[v]);
            }
        }
        const int R = static_cast<int>(m.reactions.size());
        const int C = static_cast<int>(classes.size());
        std::vector<int> change;
        std::vector<double> rates(static_cast<std::size_t>(R) * C * ntuple);
        std::vector<int> counts(S);
        for (int r = 0; r < R; ++r) {
            if (static_cast<int>(m.reactions[r].change.size()) != S) {
                throw std::invalid_argument("change vector length differs from the species count");
            }
            change.insert(change.end(), m.reactions[r].change.begin(), m.reactions[r].change.end());
            for (int c = 0; c < C; ++c) {
                for (int t = 0; t < ntuple; ++t) {
                    int rem = t;
                    for (int s = S - 1; s >= 0; --s) {
                        counts[s] = rem % (limits[s] + 1);
                        rem /= limits[s] + 1;
                    }
                    rates[(static_cast<std::size_t>(r) * C + c) * ntuple + t] =
                        m.reactions[r].rate(view<const int>(counts.data(), counts.size()), classes[c]);
                }
            }
        }
        check(mk_model_set_reactions(h, R, change.data(), limits.data(), C, C > 1 ? vclass.data() : nullptr,
                                     rates.data()));
    }
    return model;
}

} // namespace detail

// ---- generator ----------------------------------------------------------------------------

enum class boundary : std::uint8_t { reflecting, absorbing };

// Q with columns as sources, dp/dt = Q p; matrix-free on the device
namespace num {

// an assembled sparse matrix on the host in CSR (what generator::matrix() returns): each row's
// columns ascending, equal positions summed
class spmat {
  public:
    using domain_type = vec<real>;
    using codomain_type = vec<real>;
    spmat() = default;
    spmat(idx rows, idx cols, array<real> values, array<idx> columns, array<idx> row_ptr)
        : rows_(rows), cols_(cols), value_(std::move(values)), column_(std::move(columns)),
          ptr_(std::move(row_ptr)) {}
    [[nodiscard]] idx rows() const { return rows_; }
    [[nodiscard]] idx cols() const { return cols_; }
    [[nodiscard]] idx nonzeros() const { return value_.size(); }
    [[nodiscard]] const array<idx> &row_ptr() const { return ptr_; }
    [[nodiscard]] const array<idx> &columns() const { return column_; }
    [[nodiscard]] const array<real> &values() const { return value_; }
    void apply(const vec<real> &x, vec<real> &y) const {
        y.assign(rows_, 0.0);
        for (idx i = 0; i < rows_; ++i) {
            real sum = 0.0;
            for (idx k = ptr_[i]; k < ptr_[i + 1]; ++k) {
                sum += value_[k] * x[column_[k]];
            }
            y[i] = sum;
        }
    }

  private:
    idx rows_ = 0, cols_ = 0;
    array<real> value_;
    array<idx> column_;
    array<idx> ptr_;
};

// a dense row-major matrix (what fsp_solution::means() returns): m(i, j)
template <typename T>
class mat {
  public:
    mat() = default;
    mat(idx rows, idx cols, T fill = T{}) : rows_(rows), cols_(cols), data_(rows * cols, fill) {}
    [[nodiscard]] idx rows() const { return rows_; }
    [[nodiscard]] idx cols() const { return cols_; }
    T &operator()(idx i, idx j) { return data_[i * cols_ + j]; }
    const T &operator()(idx i, idx j) const { return data_[i * cols_ + j]; }
    [[nodiscard]] const array<T> &data() const { return data_; }

  private:
    idx rows_ = 0, cols_ = 0;
    array<T> data_;
};

} // namespace num

namespace detail {

// copies an assembled generator (mk_csr) to a host spmat and frees it
inline num::spmat take_csr(mk_csr m) {
    std::unique_ptr<mk_csr_s, void (*)(mk_csr)> hold(m, mk_csr_destroy);
    int64_t rows = 0, nnz = 0;
    check(mk_csr_size(m, &rows, &nnz));
    std::vector<int64_t> ptr(static_cast<std::size_t>(rows) + 1), col(static_cast<std::size_t>(nnz));
    array<real> val(static_cast<std::size_t>(nnz));
    check(mk_csr_copy_host(m, ptr.data(), col.data(), val.data()));
    return num::spmat(static_cast<idx>(rows), static_cast<idx>(rows), std::move(val),
                      array<idx>(col.begin(), col.end()), array<idx>(ptr.begin(), ptr.end()));
}

} // namespace detail

class generator {
  public:
    using domain_type = vec<real>;
    using codomain_type = vec<real>;

    // Q over any listed state space (an FSP support, a distribution) of any model that lists its
    // jumps (generator.hpp:27-44): a jump into the space is an entry, one leaving it adds to the
    // leak rate, and an absorbing boundary keeps the leak on the diagonal. The jumps are listed
    // on the host; Q is kept on the device in CSR and applied there (mk_csr_apply).
    template <state_space Space, markov_model Model>
        requires(!std::derived_from<Space, population_space>)
    generator(const Space &space, const Model &model, boundary leaks = boundary::absorbing) {
        const idx n = space.size();
        auto listed = std::make_shared<listed_jumps>();
        listed->first.assign(n + 1, 0);
        array<real> exit(n, 0.0), leak(n, 0.0);
        for (idx j = 0; j < n; ++j) {
            for (const transition &e : model.transitions(space[j])) {
                if (const std::optional<idx> i = space.find(e.to)) {
                    listed->jumps.push_back({*i, e.rate});
                    exit[j] += e.rate;
                } else {
                    leak[j] += e.rate;
                }
            }
            if (leaks == boundary::absorbing) {
                exit[j] += leak[j];
            }
            listed->first[j + 1] = listed->jumps.size();
        }
        listed->Q = assemble_listed(n, listed->first, listed->jumps, exit);
        const num::spmat &Q = listed->Q;
        std::vector<int64_t> ptr(Q.row_ptr().begin(), Q.row_ptr().end());
        std::vector<int64_t> col(Q.columns().begin(), Q.columns().end());
        mk_csr m = nullptr;
        detail::check(mk_csr_create_host(static_cast<int64_t>(n), ptr.data(), col.data(), Q.values().data(), &m));
        csr_.reset(m, [](mk_csr c) { mk_csr_destroy(c); });
        listed_ = std::move(listed);
        rates_ = std::make_shared<std::pair<array<real>, array<real>>>(std::move(exit), std::move(leak));
        n_ = n;
        if (n_ > 0) {
            x_ = std::make_shared<detail::device_vector>(n_);
            y_ = std::make_shared<detail::device_vector>(n_);
        }
    }

    template <typename Graph>
    generator(const population_space &space, const reaction_diffusion<Graph> &model,
              boundary leaks = boundary::absorbing) {
        model_ = detail::make_model(model, space.limits());
        mk_generator h = nullptr;
        detail::check(mk_generator_create(space.handle(), model_.get(),
                                          leaks == boundary::absorbing ? 1 : 0, &h));
        h_.reset(h, [](mk_generator p) { mk_generator_destroy(p); });
        int64_t n = 0;
        detail::check(mk_generator_rows(h, &n));
        n_ = static_cast<idx>(n);
        x_ = std::make_shared<detail::device_vector>(n_);
        y_ = std::make_shared<detail::device_vector>(n_);
        detail::check(mk_generator_exit_leak(h, x_->get(), y_->get(), nullptr));
        auto rates = std::make_shared<std::pair<array<real>, array<real>>>(array<real>(n_), array<real>(n_));
        x_->download(rates->first.data());
        y_->download(rates->second.data());
        rates_ = std::move(rates);
    }
    // a jump out of a state: the target's index and the rate (markovkit/generator.hpp:22-25)
    struct jump {
        idx to;
        real rate;
    };
    [[nodiscard]] idx rows() const { return n_; }
    [[nodiscard]] idx cols() const { return n_; }
    // y = Q x
    void apply(const vec<real> &x, vec<real> &y) const {
        y.resize(n_);
        if (n_ == 0) {
            return;
        }
        x_->upload(x.data());
        detail::check(csr_ ? mk_csr_apply(csr_.get(), 0.0, 1.0, x_->get(), y_->get(), nullptr)
                           : mk_generator_apply(h_.get(), x_->get(), y_->get(), nullptr));
        y_->download(y.data());
    }
    // y = shift x - Q x
    void apply_shifted(real shift, view<const real> x, view<real> y) const {
        if (n_ == 0) {
            return;
        }
        x_->upload(x.data());
        detail::check(csr_ ? mk_csr_apply(csr_.get(), shift, -1.0, x_->get(), y_->get(), nullptr)
                           : mk_generator_apply_shifted(h_.get(), shift, x_->get(), y_->get(), nullptr));
        y_->download(y.data());
    }
    // the total rate out of each state, and the part of it that leaves the space
    [[nodiscard]] const array<real> &exit_rates() const { return rates_->first; }
    [[nodiscard]] const array<real> &leak_rates() const { return rates_->second; }
    // the jumps out of state j that stay in the space, in the reference's order
    [[nodiscard]] array<jump> jumps(idx j) const {
        if (listed_) {
            return array<jump>(listed_->jumps.begin() + static_cast<std::ptrdiff_t>(listed_->first[j]),
                               listed_->jumps.begin() + static_cast<std::ptrdiff_t>(listed_->first[j + 1]));
        }
        int64_t count = 0;
        detail::check(mk_generator_jumps(h_.get(), static_cast<int64_t>(j), nullptr, nullptr, 0, &count));
        std::vector<int64_t> to(static_cast<std::size_t>(count));
        std::vector<real> rate(static_cast<std::size_t>(count));
        detail::check(mk_generator_jumps(h_.get(), static_cast<int64_t>(j), to.data(), rate.data(), count, &count));
        array<jump> out(static_cast<std::size_t>(count));
        for (std::size_t k = 0; k < out.size(); ++k) {
            out[k] = {static_cast<idx>(to[k]), rate[k]};
        }
        return out;
    }
    [[nodiscard]] idx n_jumps() const {
        if (listed_) {
            return listed_->jumps.size();
        }
        int64_t n = 0;
        detail::check(mk_generator_n_jumps(h_.get(), &n, nullptr));
        return static_cast<idx>(n);
    }
    // Q, assembled
    [[nodiscard]] num::spmat matrix() const {
        if (listed_) {
            return listed_->Q;
        }
        mk_csr m = nullptr;
        detail::check(mk_generator_matrix(h_.get(), &m, nullptr));
        return detail::take_csr(m);
    }
    // shift I - Q, assembled
    [[nodiscard]] num::spmat characteristic_matrix(real shift) const {
        if (listed_) {
            const num::spmat &Q = listed_->Q;
            array<real> v(Q.values().size());
            for (idx i = 0; i < Q.rows(); ++i) {
                for (idx k = Q.row_ptr()[i]; k < Q.row_ptr()[i + 1]; ++k) {
                    v[k] = (Q.columns()[k] == i ? shift : 0.0) - Q.values()[k];
                }
            }
            return num::spmat(Q.rows(), Q.cols(), std::move(v), Q.columns(), Q.row_ptr());
        }
        mk_csr m = nullptr;
        detail::check(mk_generator_characteristic_matrix(h_.get(), shift, &m, nullptr));
        return detail::take_csr(m);
    }
    // the device handle of a population-space generator (null for one over a listed space)
    [[nodiscard]] mk_generator handle() const { return h_.get(); }
    [[nodiscard]] mk_model model_handle() const { return model_.get(); }
    // the device CSR of a generator over a listed space (null for a population-space one)
    [[nodiscard]] mk_csr csr_handle() const { return csr_.get(); }

  private:
    struct listed_jumps {
        array<idx> first;  // jumps out of state j: [first[j], first[j + 1])
        array<jump> jumps;
        num::spmat Q;      // rows are targets: Q[to][from] = rate, Q[j][j] = -exit[j]
    };

    // Q in CSR from the jumps: each row's columns ascending, equal positions summed
    static num::spmat assemble_listed(idx n, const array<idx> &first, const array<jump> &jumps,
                                      const array<real> &exit) {
        array<array<std::pair<idx, real>>> rows(n);
        for (idx j = 0; j < n; ++j) {
            rows[j].push_back({j, -exit[j]});
            for (idx k = first[j]; k < first[j + 1]; ++k) {
                rows[jumps[k].to].push_back({j, jumps[k].rate});
            }
        }
        array<idx> ptr(n + 1, 0), col;
        array<real> val;
        for (idx i = 0; i < n; ++i) {
            auto &r = rows[i];
            std::stable_sort(r.begin(), r.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
            for (const auto &[c, v] : r) {
                if (!col.empty() && static_cast<idx>(col.size()) > ptr[i] && col.back() == c) {
                    val.back() += v;
                } else {
                    col.push_back(c);
                    val.push_back(v);
                }
            }
            ptr[i + 1] = col.size();
        }
        return num::spmat(n, n, std::move(val), std::move(col), std::move(ptr));
    }

    std::shared_ptr<const listed_jumps> listed_;
    std::shared_ptr<mk_csr_s> csr_;
    std::shared_ptr<mk_model_s> model_;
    std::shared_ptr<const std::pair<array<real>, array<real>>> rates_; // exit, leak
    std::shared_ptr<mk_generator_s> h_;
    std::shared_ptr<detail::device_vector> x_, y_;
    idx n_ = 0;
};

// shift I - Q; reads Q by reference (the reference keeps a pointer too)
class shifted_generator {
  public:
    using domain_type = vec<real>;
    using codomain_type = vec<real>;
    shifted_generator(const generator &Q, real shift) : Q_(&Q), shift_(shift) {}
    [[nodiscard]] idx rows() const { return Q_->rows(); }
    [[nodiscard]] idx cols() const { return Q_->cols(); }
    [[nodiscard]] real shift() const { return shift_; }
    [[nodiscard]] const generator &base() const { return *Q_; }
    void apply(const vec<real> &x, vec<real> &y) const {
        y.resize(rows());
        Q_->apply_shifted(shift_, view<const real>(x.data(), x.size()), view<real>(y.data(), y.size()));
    }
    [[nodiscard]] num::spmat matrix() const { return Q_->characteristic_matrix(shift_); }

  private:
    const generator *Q_;
    real shift_;
};

// ---- multigrid ----------------------------------------------------------------------------

// multigrid.hpp:120-123, with this library's two other smoothers after the reference's two
enum class relaxation : std::uint8_t {
    jacobi,          // weighted point Jacobi
    aggregate_block, // exact solves on states that differ only inside one coarse voxel
    gauss_seidel,    // red-black Gauss-Seidel
    ilu0             // red-black ILU(0)
};

struct multigrid_options {
    int pre_sweeps = 2;
    int post_sweeps = 2;
    real jacobi_weight = 2.0 / 3.0;
    idx coarsest_size = 4;
    int max_levels = 32;
    int coarse_cycles = 1;
    int sweep_growth = 0;
    relaxation smoother = relaxation::jacobi;
    int precision = 0; // 0 FP64, 1 FP32 (use with flexible GMRES)
};

namespace detail {

inline mk_multigrid_options to_c(const multigrid_options &o) {
    mk_multigrid_options c{};
    mk_multigrid_options_default(&c);
    c.pre_sweeps = o.pre_sweeps;
    c.post_sweeps = o.post_sweeps;
    c.jacobi_weight = o.jacobi_weight;
    c.coarsest_size = static_cast<int64_t>(o.coarsest_size);
    c.max_levels = o.max_levels;
    c.coarse_cycles = o.coarse_cycles;
    c.sweep_growth = o.sweep_growth;
    static constexpr int kSmoother[] = {0, 3, 1, 2}; // the C ABI's numbering
    c.smoother = kSmoother[static_cast<int>(o.smoother)];
    c.precision = o.precision;
    return c;
}

} // namespace detail

// The reference's sector_multigrid<D> (markovkit/rdme/multigrid.hpp:364-408), over a grid<D>
// domain; CTAD takes D from the domain. Copies share one device hierarchy.
template <int D>
class sector_multigrid {
  public:
    using domain_type = vec<real>;
    using codomain_type = vec<real>;

    sector_multigrid(const voxel_domain<grid<D>> &domain, const population_box &box, real shift,
                     const multigrid_options &options = {}) {
        init(reaction_diffusion<grid<D>>{domain, {}}, box, shift, options);
    }
    sector_multigrid(const voxel_domain<grid<D>> &domain, const population_sector &sector, real shift,
                     const multigrid_options &options = {}) {
        init(reaction_diffusion<grid<D>>{domain, {}}, sector, shift, options);
    }
    [[nodiscard]] idx rows() const { return n_; }
    [[nodiscard]] idx cols() const { return n_; }
    [[nodiscard]] idx n_sectors() const { return sectors_; }
    [[nodiscard]] std::size_t max_levels() const {
        int l = 0;
        detail::check(mk_multigrid_max_levels(h_.get(), &l));
        return static_cast<std::size_t>(l);
    }
    // one cycle per sector from a zero initial guess: x = M b
    void apply(const vec<real> &b, vec<real> &x) const {
        b_->upload(b.data());
        detail::check(mk_multigrid_apply(h_.get(), b_->get(), x_->get(), nullptr));
        x.resize(n_);
        x_->download(x.data());
    }
    [[nodiscard]] mk_multigrid handle() const { return h_.get(); }
    [[nodiscard]] bool fp32() const { return fp32_; }

  protected:
    sector_multigrid() = default;
    void init(const reaction_diffusion<grid<D>> &m, const population_space &space, real shift,
              const multigrid_options &o) {
        auto model = detail::make_model(m, space.limits());
        const mk_multigrid_options c = detail::to_c(o);
        mk_multigrid h = nullptr;
        detail::check(mk_multigrid_create(space.handle(), model.get(), shift, &c, &h));
        h_.reset(h, [](mk_multigrid p) { mk_multigrid_destroy(p); });
        n_ = space.size();
        sectors_ = space.n_sectors();
        fp32_ = o.precision == 1;
        b_ = std::make_shared<detail::device_vector>(n_);
        x_ = std::make_shared<detail::device_vector>(n_);
    }
    std::shared_ptr<mk_multigrid_s> h_;
    std::shared_ptr<detail::device_vector> b_, x_;
    idx n_ = 0, sectors_ = 0;
    bool fp32_ = false;
};

// one depth of a population_multigrid hierarchy: y = A_d x
class population_multigrid_level {
  public:
    population_multigrid_level(std::shared_ptr<mk_multigrid_s> h, int depth, idx n)
        : h_(std::move(h)), depth_(depth), n_(n), x_(std::make_shared<detail::device_vector>(n)),
          y_(std::make_shared<detail::device_vector>(n)) {}
    [[nodiscard]] idx rows() const { return n_; }
    [[nodiscard]] idx cols() const { return n_; }
    void apply_system(view<const real> x, view<real> y) const {
        x_->upload(x.data());
        detail::check(mk_multigrid_apply_system(h_.get(), depth_, x_->get(), y_->get(), nullptr));
        y_->download(y.data());
    }

  private:
    std::shared_ptr<mk_multigrid_s> h_;
    int depth_ = 0;
    idx n_ = 0;
    std::shared_ptr<detail::device_vector> x_, y_;
};

// population_transfer between depth d and d + 1 (multigrid.hpp:48-111)
class population_transfer_view {
  public:
    population_transfer_view(std::shared_ptr<mk_multigrid_s> h, int depth, idx fine, idx coarse)
        : h_(std::move(h)), depth_(depth), fine_(fine), coarse_(coarse),
          f_(std::make_shared<detail::device_vector>(fine)),
          c_(std::make_shared<detail::device_vector>(coarse)) {}
    [[nodiscard]] idx fine_size() const { return fine_; }
    [[nodiscard]] idx coarse_size() const { return coarse_; }
    // coarse[c(i)] += fine[i], in a fixed order
    void restrict(view<const real> fine, view<real> coarse) const {
        f_->upload(fine.data());
        detail::check(mk_multigrid_restrict(h_.get(), depth_, f_->get(), c_->get(), nullptr));
        c_->download(coarse.data());
    }
    // fine[i] = w_i coarse[c(i)]
    void prolong(view<const real> coarse, view<real> fine) const {
        c_->upload(coarse.data());
        detail::check(mk_multigrid_prolong(h_.get(), depth_, c_->get(), f_->get(), nullptr));
        f_->download(fine.data());
    }

  private:
    std::shared_ptr<mk_multigrid_s> h_;
    int depth_ = 0;
    idx fine_ = 0, coarse_ = 0;
    std::shared_ptr<detail::device_vector> f_, c_;
};

// The reference's population_multigrid<D> (multigrid.hpp:136-361): the multigrid of one
// population sector of a diffusion-only grid model, as its own object with its levels and
// transfers exposed (the device hierarchy is the sector multigrid's, on that one sector)
template <int D>
class population_multigrid : public sector_multigrid<D> {
  public:
    population_multigrid(const voxel_domain<grid<D>> &domain, const array<int> &totals, real shift,
                         multigrid_options options = {})
        : domain_(domain), totals_(totals), shift_(shift) {
        const population_sector space(domain.n_voxels(), totals);
        this->init(reaction_diffusion<grid<D>>{domain, {}}, space, shift, options);
        int depth = 0;
        detail::check(mk_multigrid_depth(this->h_.get(), &depth));
        for (int d = 0; d < depth; ++d) {
            int64_t n = 0;
            detail::check(mk_multigrid_level_size(this->h_.get(), d, &n));
            sizes_.push_back(static_cast<idx>(n));
        }
        for (int d = 0; d < depth; ++d) {
            levels_.push_back(std::make_shared<population_multigrid_level>(this->h_, d, sizes_[d]));
            if (d + 1 < depth) {
                transfers_.push_back(std::make_shared<population_transfer_view>(this->h_, d, sizes_[d],
                                                                                sizes_[d + 1]));
            }
        }
    }
    [[nodiscard]] real shift() const { return shift_; }
    [[nodiscard]] idx n_levels() const { return sizes_.size(); }
    // y = (shift I - Q) x on this level's sector
    void apply_system(view<const real> x, view<real> y) const { levels_.front()->apply_system(x, y); }
    [[nodiscard]] const population_transfer_view &transfer() const {
        if (transfers_.empty()) {
            throw std::logic_error("population_multigrid: a single level has no transfer");
        }
        return *transfers_.front();
    }
    [[nodiscard]] const population_multigrid_level *coarse_level() const {
        return levels_.size() > 1 ? levels_[1].get() : nullptr;
    }
    // states of every level over those of the finest
    [[nodiscard]] real grid_complexity() const {
        real total = 0.0;
        for (idx n : sizes_) {
            total += static_cast<real>(n);
        }
        return total / static_cast<real>(sizes_.front());
    }
    // entries (states plus jumps) of every level's operator over those of the finest; each
    // level's jumps are counted on its own diffusion-only generator
    [[nodiscard]] real operator_complexity() const {
        real total = 0.0, fine = 0.0;
        std::array<idx, D> dims = domain_.graph.dims;
        std::array<real, D> spacing = domain_.graph.spacing;
        for (idx d = 0; d < sizes_.size(); ++d) {
            const voxel_domain<grid<D>> dom(grid<D>(dims, spacing), domain_.diffusivities);
            const population_sector space(dom.n_voxels(), totals_);
            const reaction_diffusion<grid<D>> model{dom, {}};
            auto h = detail::make_model(model, space.limits());
            mk_generator g = nullptr;
            detail::check(mk_generator_create(space.handle(), h.get(), 1, &g));
            std::unique_ptr<mk_generator_s, void (*)(mk_generator)> hold(g, mk_generator_destroy);
            int64_t jumps = 0;
            detail::check(mk_generator_n_jumps(g, &jumps, nullptr));
            const real entries = static_cast<real>(space.size()) + static_cast<real>(jumps);
            total += entries;
            if (d == 0) {
                fine = entries;
            }
            for (int a = 0; a < D; ++a) {
                if (dims[a] > 1) {
                    dims[a] /= 2;
                    spacing[a] *= 2.0;
                }
            }
        }
        return total / fine;
    }

  private:
    voxel_domain<grid<D>> domain_;
    array<int> totals_;
    real shift_ = 0.0;
    array<idx> sizes_;
    array<std::shared_ptr<population_multigrid_level>> levels_;
    array<std::shared_ptr<population_transfer_view>> transfers_;
};

template <int D>
population_multigrid(const voxel_domain<grid<D>> &, const array<int> &, real) -> population_multigrid<D>;
template <int D>
population_multigrid(const voxel_domain<grid<D>> &, const array<int> &, real, multigrid_options)
    -> population_multigrid<D>;

// ---- preconditioners and GMRES -------------------------------------------------------------

namespace num {

template <typename Op, typename X, typename Y>
concept linear_operator = requires(const Op &A, const X &x, Y &y) {
    { A.rows() } -> std::convertible_to<idx>;
    { A.cols() } -> std::convertible_to<idx>;
    A.apply(x, y);
};

namespace detail {

// a preconditioner handle of the C ABI shared by copies, with a host apply(x, y)
class device_preconditioner {
  public:
    [[nodiscard]] idx rows() const { return n_; }
    [[nodiscard]] idx cols() const { return n_; }
    void apply(const vec<real> &x, vec<real> &y) const {
        if (x.size() != n_) {
            throw std::invalid_argument("preconditioner: vector size differs from the operator's");
        }
        x_->upload(x.data());
        markovkit::detail::check(mk_precond_apply(h_.get(), x_->get(), y_->get(), nullptr));
        y.resize(n_);
        y_->download(y.data());
    }
    [[nodiscard]] mk_precond precond_handle() const { return h_.get(); }

  protected:
    void adopt(mk_precond h) {
        h_.reset(h, [](mk_precond p) { mk_precond_destroy(p); });
        int64_t n = 0;
        markovkit::detail::check(mk_precond_size(h, &n));
        n_ = static_cast<idx>(n);
        x_ = std::make_shared<markovkit::detail::device_vector>(n_);
        y_ = std::make_shared<markovkit::detail::device_vector>(n_);
    }

  private:
    std::shared_ptr<mk_precond_s> h_;
    std::shared_ptr<markovkit::detail::device_vector> x_, y_;
    idx n_ = 0;
};

} // namespace detail

// z = d .* v with d the given inverse diagonal (num::jacobi_preconditioner)
class jacobi_preconditioner : public detail::device_preconditioner {
  public:
    explicit jacobi_preconditioner(vec<real> inverse_diagonal) {
        mk_precond h = nullptr;
        markovkit::detail::check(mk_precond_create_diagonal(
            static_cast<int64_t>(inverse_diagonal.size()), inverse_diagonal.data(), &h));
        adopt(h);
    }
};

// ILU(0) of an assembled matrix in its row order (num::ilu0_preconditioner), factored and
// applied on the device
class ilu0_preconditioner : public detail::device_preconditioner {
  public:
    explicit ilu0_preconditioner(const spmat &A) {
        if (A.rows() != A.cols()) {
            throw std::invalid_argument("ilu0_preconditioner: the matrix must be square");
        }
        const std::vector<int64_t> ptr(A.row_ptr().begin(), A.row_ptr().end());
        const std::vector<int64_t> col(A.columns().begin(), A.columns().end());
        mk_precond h = nullptr;
        markovkit::detail::check(mk_precond_create_ilu0(static_cast<int64_t>(A.rows()), ptr.data(),
                                                        col.data(), A.values().data(), nullptr, &h));
        adopt(h);
    }
    // depth of the forward and backward level sets, and launches per application
    [[nodiscard]] std::array<idx, 3> schedule() const {
        int64_t lo = 0, up = 0, launches = 0;
        markovkit::detail::check(mk_precond_ilu0_schedule(precond_handle(), &lo, &up, &launches));
        return {static_cast<idx>(lo), static_cast<idx>(up), static_cast<idx>(launches)};
    }
};

struct gmres_options {
    real tolerance = 1e-8; // absolute, on ||b - A x||_2
    idx max_iterations = 1000;
    idx restart = 30;
};

struct solver_result {
    idx iterations = 0;
    real residual = 0.0;
    bool converged = false;
};

namespace detail {

inline solver_result run(const shifted_generator &A, mk_multigrid mg, mk_precond pc,
                         const vec<real> &b, vec<real> &x, const gmres_options &o) {
    if (b.size() != A.rows() || x.size() != A.rows()) {
        throw std::invalid_argument("gmres: vector sizes differ from the operator's");
    }
    mk_gmres_options c{};
    mk_gmres_options_default(&c);
    c.tolerance = o.tolerance;
    c.max_iterations = static_cast<int64_t>(o.max_iterations);
    c.restart = static_cast<int>(std::min<idx>(o.restart, 1u << 30));
    mk_solver h = nullptr;
    if (pc) {
        markovkit::detail::check(mk_solver_create_pc(A.base().handle(), A.shift(), pc, &c, &h));
    } else {
        markovkit::detail::check(mk_solver_create(A.base().handle(), A.shift(), mg, &c, &h));
    }
    std::unique_ptr<mk_solver_s, void (*)(mk_solver)> solver(h, [](mk_solver p) { mk_solver_destroy(p); });
    mk_solver_result r{};
    const int rc = mk_solver_solve_host(h, b.data(), x.data(), &r, nullptr);
    if (rc != MK_OK && rc != MK_ENOTCONV) {
        markovkit::detail::check(rc);
    }
    return {static_cast<idx>(r.iterations), r.residual, r.converged != 0};
}

// a host operator as a preconditioner handle: each application copies v out, calls
// M.apply(v, z) on the calling thread and copies z back
template <typename M>
int host_apply(void *ctx, const double *v, double *z, int64_t n) {
    try {
        const auto &op = *static_cast<const M *>(ctx);
        const vec<real> in(v, v + n);
        vec<real> out(static_cast<std::size_t>(n), 0.0);
        op.apply(in, out);
        if (out.size() != static_cast<std::size_t>(n)) {
            return 1;
        }
        std::copy(out.begin(), out.end(), z);
        return 0;
    } catch (...) {
        return 1;
    }
}

} // namespace detail

// restarted GMRES on A = shift I - Q; x holds the initial guess and the solution
inline solver_result gmres(const shifted_generator &A, const vec<real> &b, vec<real> &x,
                           const gmres_options &options = {}) {
    return detail::run(A, nullptr, nullptr, b, x, options);
}

// right-preconditioned by a sector multigrid (flexible GMRES when it runs in FP32)
template <int D>
solver_result gmres(const shifted_generator &A, const sector_multigrid<D> &M, const vec<real> &b,
                    vec<real> &x, const gmres_options &options = {}) {
    return detail::run(A, M.handle(), nullptr, b, x, options);
}

// right-preconditioned by a device preconditioner (jacobi_preconditioner, ilu0_preconditioner)
// or by any other operator with rows() and apply(x, y), applied on the host
template <typename M>
    requires linear_operator<M, vec<real>, vec<real>>
solver_result gmres(const shifted_generator &A, const M &pre, const vec<real> &b, vec<real> &x,
                    const gmres_options &options = {}) {
    if constexpr (requires { pre.precond_handle(); }) {
        return detail::run(A, nullptr, pre.precond_handle(), b, x, options);
    } else {
        if (pre.rows() != A.rows()) {
            throw std::invalid_argument("gmres: preconditioner size differs from the operator's");
        }
        mk_precond h = nullptr;
        markovkit::detail::check(mk_precond_create_host(static_cast<int64_t>(A.rows()),
                                                        &detail::host_apply<M>,
                                                        const_cast<M *>(&pre), &h));
        std::unique_ptr<mk_precond_s, void (*)(mk_precond)> hold(h, [](mk_precond p) { mk_precond_destroy(p); });
        return detail::run(A, nullptr, h, b, x, options);
    }
}

} // namespace num

// ---- Krylov FSP ---------------------------------------------------------------------------

struct reaction {
    state change;
    std::function<real(const state &)> rate;
};

struct reaction_network {
    array<reaction> reactions;

    // every reaction with a positive rate whose result has no negative count
    // (reaction_network.hpp:20-37); host-side, for callers that enumerate jumps
    [[nodiscard]] array<transition> transitions(const state &x) const {
        array<transition> result;
        for (const reaction &r : reactions) {
            const real rate = r.rate(x);
            if (!(rate > 0.0)) {
                continue;
            }
            state y = x;
            bool valid = true;
            for (idx s = 0; s < y.size(); ++s) {
                y[s] += r.change[s];
                valid = valid && y[s] >= 0;
            }
            if (valid) {
                result.push_back({std::move(y), rate});
            }
        }
        return result;
    }
};

// the states an FSP may add to its support (fsp.hpp:16-42): box(bounds), box(bound) and
// everywhere() run on the device; a region made from any other predicate serves the host-side
// expand() and generator only. The default region is everywhere(), as in the reference.
class region {
  public:
    region() = default;
    template <typename F>
        requires(!std::same_as<std::decay_t<F>, region> && std::is_invocable_r_v<bool, const F &, const state &>)
    region(F f) : kind_(kind::predicate), predicate_(std::move(f)) {}

    static region bounded(array<int> bounds) {
        region r;
        r.kind_ = kind::box;
        r.bounds_ = std::move(bounds);
        return r;
    }
    static region uniform(int bound) {
        region r;
        r.kind_ = kind::uniform;
        r.uniform_ = bound;
        return r;
    }

    [[nodiscard]] bool operator()(const state &x) const {
        switch (kind_) {
        case kind::everywhere:
            return true;
        case kind::predicate:
            return predicate_(x);
        case kind::uniform:
            return std::all_of(x.begin(), x.end(), [&](int c) { return c >= 0 && c <= uniform_; });
        case kind::box:
            break;
        }
        for (idx s = 0; s < x.size(); ++s) {
            if (s >= bounds_.size() || x[s] < 0 || x[s] > bounds_[s]) {
                return false;
            }
        }
        return true;
    }
    [[nodiscard]] bool is_everywhere() const { return kind_ == kind::everywhere; }
    [[nodiscard]] bool is_box() const { return kind_ == kind::box || kind_ == kind::uniform; }
    // the box's bounds over `species` species
    [[nodiscard]] array<int> bounds(idx species) const {
        if (kind_ == kind::uniform) {
            return array<int>(species, uniform_);
        }
        if (kind_ != kind::box || bounds_.size() != species) {
            throw std::invalid_argument("fsp: the region is not a box over every species");
        }
        return bounds_;
    }

  private:
    enum class kind : std::uint8_t { everywhere, box, uniform, predicate };
    kind kind_ = kind::everywhere;
    array<int> bounds_;
    int uniform_ = 0;
    std::function<bool(const state &)> predicate_;
};

// 0 <= x[s] <= bounds[s] for every coordinate (fsp.hpp:26-35)
inline region box(array<int> bounds) { return region::bounded(std::move(bounds)); }
// 0 <= x[s] <= bound for every coordinate (fsp.hpp:37-42)
inline region box(int bound) { return region::uniform(bound); }
inline region everywhere() { return region{}; }

struct krylov_fsp_options {
    region inside = everywhere();
    real tolerance = 1e-6;
    real initial_step = 1.0;
    real step_growth = 2.0;
    real drop_probability = 1e-10;
    real drop_derivative = 1e-16;
    int layers = 1;
    int save_every = 1000; // accepted for source compatibility; only the final state is saved
    int max_steps = 1 << 28;
    int krylov_dim = 30;
    real krylov_tol = 1e-8;
};

// adaptive_fsp_options (fsp.hpp:108-121); sampled_expansion has no device counterpart
struct adaptive_fsp_options {
    region inside = everywhere();
    real step_scale = 1.0;
    real prune_fraction = 0.1;
    real flux_tolerance = 1e-6;
    real min_probability = 0.0;
    int layers = 1;
    bool sampled_expansion = false;
    unsigned seed = 42;
    int save_every = 1000; // accepted for source compatibility; only the final state is saved
    int max_steps = 1 << 28;
    int krylov_dim = 30;
    real krylov_tol = 1e-8;
};

// states, their probabilities and a lookup from state to index (distribution.hpp:10-88); a
// state_space, so generator(p, model, boundary) lists Q over it
class distribution {
  public:
    distribution() = default;
    // the point mass at x
    explicit distribution(const state &x) { add(x, 1.0); }
    distribution(array<state> states, array<real> p) : states_(std::move(states)), p_(std::move(p)) {
        for (idx i = 0; i < states_.size(); ++i) {
            index_.emplace(states_[i], i);
        }
    }
    [[nodiscard]] idx size() const { return states_.size(); }
    [[nodiscard]] const state &operator[](idx i) const { return states_[i]; }
    [[nodiscard]] const array<state> &states() const { return states_; }
    [[nodiscard]] array<real> &probabilities() { return p_; }
    [[nodiscard]] const array<real> &probabilities() const { return p_; }
    [[nodiscard]] std::optional<idx> find(const state &x) const {
        const auto it = index_.find(x);
        return it == index_.end() ? std::nullopt : std::optional<idx>(it->second);
    }
    // x with probability `mass`, unless x is already present
    void add(const state &x, real mass = 0.0) {
        if (index_.emplace(x, states_.size()).second) {
            states_.push_back(x);
            p_.push_back(mass);
        }
    }
    // drops every state i with remove(i); the others keep their order
    template <typename Remove>
    void remove_if(Remove remove) {
        array<bool> gone(size());
        for (idx i = 0; i < size(); ++i) {
            gone[i] = static_cast<bool>(remove(i));
        }
        idx n = 0;
        for (idx i = 0; i < size(); ++i) {
            if (!gone[i]) {
                if (n != i) {
                    states_[n] = std::move(states_[i]);
                    p_[n] = p_[i];
                }
                ++n;
            }
        }
        states_.resize(n);
        p_.resize(n);
        index_.clear();
        for (idx i = 0; i < n; ++i) {
            index_.emplace(states_[i], i);
        }
    }
    // negative entries (roundoff) become 0, then the total is scaled to 1; returns the total
    // before scaling
    real normalize() {
        real total = 0.0;
        for (real &v : p_) {
            v = v < 0.0 ? 0.0 : v;
            total += v;
        }
        if (total > 0.0) {
            for (real &v : p_) {
                v /= total;
            }
        }
        return total;
    }
    [[nodiscard]] vec<real> means() const {
        vec<real> m(states_.empty() ? 0 : states_.front().size(), 0.0);
        for (idx i = 0; i < size(); ++i) {
            for (idx s = 0; s < m.size(); ++s) {
                m[s] += p_[i] * states_[i][s];
            }
        }
        return m;
    }
    [[nodiscard]] std::map<int, real> marginal(idx s) const {
        std::map<int, real> out;
        for (idx i = 0; i < size(); ++i) {
            out[states_[i][s]] += p_[i];
        }
        return out;
    }

  private:
    array<state> states_;
    array<real> p_;
    std::map<state, idx> index_;
};

// adds `layers` rings of neighbours inside the region; a ring after the first grows only from
// the states the ring before added (fsp.hpp:44-59). Host-side, for callers that build a support.
template <markov_model Model>
void expand(distribution &p, const Model &model, const region &inside, int layers = 1) {
    idx from = 0;
    for (int layer = 0; layer < layers; ++layer) {
        const idx to = p.size();
        for (idx i = from; i < to; ++i) {
            for (const transition &e : model.transitions(p[i])) {
                if (inside(e.to)) {
                    p.add(e.to);
                }
            }
        }
        from = to;
    }
}

struct fsp_solution {
    array<real> times;
    array<distribution> snapshots;
    // means(k, s): the mean count of species s at times[k] (fsp.hpp:90-101)
    [[nodiscard]] num::mat<real> means() const {
        const idx species = snapshots.empty() || snapshots.front().size() == 0 ? 0 : snapshots.front()[0].size();
        num::mat<real> m(snapshots.size(), species, 0.0);
        for (idx k = 0; k < snapshots.size(); ++k) {
            const vec<real> v = snapshots[k].means();
            for (idx s = 0; s < species && s < v.size(); ++s) {
                m(k, s) = v[s];
            }
        }
        return m;
    }
};

namespace detail {

struct fsp_tables {
    array<int> bounds, change, initial;
    array<real> rates;
    idx box = 1;
};

// the network's propensities over box(bounds), box order (species 0 most significant)
inline fsp_tables tabulate(const reaction_network &model, const state &initial, const array<int> &bounds) {
    fsp_tables t;
    t.bounds = bounds;
    const idx S = t.bounds.size();
    if (S == 0 || S != initial.size()) {
        throw std::invalid_argument("fsp: the box must bound every species");
    }
    for (int b : t.bounds) {
        t.box *= static_cast<idx>(b) + 1;
    }
    const idx R = model.reactions.size();
    t.rates.assign(R * t.box, 0.0);
    state x(S);
    for (idx i = 0; i < t.box; ++i) {
        idx rem = i;
        for (idx s = S; s-- > 0;) {
            x[s] = static_cast<int>(rem % (t.bounds[s] + 1));
            rem /= t.bounds[s] + 1;
        }
        for (idx r = 0; r < R; ++r) {
            t.rates[r * t.box + i] = model.reactions[r].rate(x);
        }
    }
    for (const auto &rx : model.reactions) {
        if (rx.change.size() != S) {
            throw std::invalid_argument("fsp: change vector length differs from the species count");
        }
        t.change.insert(t.change.end(), rx.change.begin(), rx.change.end());
    }
    t.initial = initial;
    return t;
}

inline void fill_options(mk_fsp_options &c, const krylov_fsp_options &o) {
    c.tolerance = o.tolerance;
    c.initial_step = o.initial_step;
    c.step_growth = o.step_growth;
    c.drop_probability = o.drop_probability;
    c.drop_derivative = o.drop_derivative;
    c.layers = o.layers;
    c.krylov_dim = o.krylov_dim;
    c.max_steps = o.max_steps;
    c.krylov_tol = o.krylov_tol;
}

inline void fill_options(mk_fsp_options &c, const adaptive_fsp_options &o) {
    if (o.sampled_expansion) {
        throw std::invalid_argument("solve_adaptive_fsp: the device expands every neighbour");
    }
    c.method = 1;
    c.step_scale = o.step_scale;
    c.prune_fraction = o.prune_fraction;
    c.flux_tolerance = o.flux_tolerance;
    c.min_probability = o.min_probability;
    c.layers = o.layers;
    c.krylov_dim = o.krylov_dim;
    c.max_steps = o.max_steps;
    c.krylov_tol = o.krylov_tol;
}

template <typename Options>
mk_fsp_problem problem(const fsp_tables &t, const reaction_network &model, real T, const Options &o) {
    mk_fsp_problem p{};
    p.n_species = static_cast<int>(t.bounds.size());
    p.n_reactions = static_cast<int>(model.reactions.size());
    p.bounds = t.bounds.data();
    p.change = t.change.data();
    p.rates = t.rates.data();
    p.initial = t.initial.data();
    p.final_time = T;
    mk_fsp_options_default(&p.options);
    fill_options(p.options, o);
    return p;
}

// the box an everywhere() instance starts in
inline array<int> first_box(const state &initial) {
    array<int> b(initial.size());
    for (idx s = 0; s < initial.size(); ++s) {
        b[s] = std::max(2 * initial[s], initial[s] + 16);
    }
    return b;
}

constexpr idx kLargestAutoBox = idx(1) << 26;

// Every instance in one launch of the batched FSP kernel. A region other than a box must be
// everywhere(): such an instance runs in a box whose bounds double (2b + 1) on each species
// an expansion would have crossed, and runs again until no expansion met the box; the support
// then grew exactly as an unbounded region lets it, so the result is the everywhere() one.
template <typename Options>
array<fsp_solution> solve_batch(const array<std::tuple<reaction_network, state, real, Options>> &instances) {
    const idx n = instances.size();
    array<array<int>> bounds(n);
    array<bool> automatic(n, false);
    for (idx k = 0; k < n; ++k) {
        const auto &[model, initial, T, o] = instances[k];
        if (o.inside.is_box()) {
            bounds[k] = o.inside.bounds(initial.size());
        } else if (o.inside.is_everywhere()) {
            automatic[k] = true;
            bounds[k] = first_box(initial);
        } else {
            throw std::invalid_argument("fsp: the device FSP takes box(...) or everywhere() as the region");
        }
    }
    array<fsp_solution> sols(n);
    array<idx> pending(n);
    for (idx k = 0; k < n; ++k) {
        pending[k] = k;
    }
    while (!pending.empty()) {
        array<fsp_tables> tables;
        array<mk_fsp_problem> problems;
        tables.reserve(pending.size());
        for (idx k : pending) {
            const auto &[model, initial, T, o] = instances[k];
            tables.push_back(tabulate(model, initial, bounds[k]));
        }
        for (idx q = 0; q < pending.size(); ++q) {
            const auto &[model, initial, T, o] = instances[pending[q]];
            problems.push_back(problem(tables[q], model, T, o));
        }
        idx total = 0;
        for (const auto &t : tables) {
            total += t.box;
        }
        array<real> out(total);
        array<mk_fsp_result> results(pending.size());
        const int rc = mk_fsp_krylov_batch(static_cast<int>(problems.size()), problems.data(), out.data(),
                                           results.data(), nullptr);
        if (rc != MK_OK && rc != MK_ENOTCONV) {
            markovkit::detail::check(rc);
        }
        array<idx> again;
        idx off = 0;
        for (idx q = 0; q < pending.size(); ++q) {
            const idx k = pending[q];
            const auto &t = tables[q];
            const idx S = t.bounds.size();
            if (automatic[k] && results[q].clipped != 0) {
                idx size = 1;
                for (idx s = 0; s < S; ++s) {
                    if (results[q].clipped & (1 << s)) {
                        bounds[k][s] = 2 * bounds[k][s] + 1;
                    }
                    size *= static_cast<idx>(bounds[k][s]) + 1;
                }
                if (size > kLargestAutoBox) {
                    throw std::runtime_error("fsp: the everywhere() support outgrew a box of 2^26 states");
                }
                again.push_back(k);
                off += t.box;
                continue;
            }
            array<state> states;
            array<real> p;
            for (idx i = 0; i < t.box; ++i) {
                if (out[off + i] != 0.0) {
                    state x(S);
                    idx rem = i;
                    for (idx s = S; s-- > 0;) {
                        x[s] = static_cast<int>(rem % (t.bounds[s] + 1));
                        rem /= t.bounds[s] + 1;
                    }
                    states.push_back(std::move(x));
                    p.push_back(out[off + i]);
                }
            }
            fsp_solution &sol = sols[k];
            sol.times = {0.0, results[q].time};
            sol.snapshots.clear();
            sol.snapshots.emplace_back(array<state>{t.initial}, array<real>{1.0});
            sol.snapshots.emplace_back(std::move(states), std::move(p));
            off += t.box;
        }
        pending = std::move(again);
    }
    return sols;
}

} // namespace detail

// solve_krylov_fsp for several instances in one launch
inline array<fsp_solution> solve_krylov_fsp_batch(
    const array<std::tuple<reaction_network, state, real, krylov_fsp_options>> &instances) {
    return detail::solve_batch(instances);
}

// solve_adaptive_fsp for several instances in one launch
inline array<fsp_solution> solve_adaptive_fsp_batch(
    const array<std::tuple<reaction_network, state, real, adaptive_fsp_options>> &instances) {
    return detail::solve_batch(instances);
}

// FSP with flux-controlled steps on the GPU (fsp.hpp:123-188)
inline fsp_solution solve_adaptive_fsp(const reaction_network &model, const state &initial,
                                       real final_time, const adaptive_fsp_options &options = {}) {
    return solve_adaptive_fsp_batch({{model, initial, final_time, options}}).front();
}

// the Krylov FSP of Vo and Sidje on the GPU (fsp.hpp:207-254)
inline fsp_solution solve_krylov_fsp(const reaction_network &model, const state &initial,
                                     real final_time, const krylov_fsp_options &options = {}) {
    return solve_krylov_fsp_batch({{model, initial, final_time, options}}).front();
}

// ---- stochastic simulation ----------------------------------------------------------------

// a piecewise-constant path: the chain is in states[k] from times[k] until times[k + 1]
// (ssa.hpp:14-39)
struct trajectory {
    array<real> times;
    array<state> states;
    [[nodiscard]] vec<real> component(idx species) const {
        vec<real> out(states.size());
        for (idx k = 0; k < states.size(); ++k) {
            out[k] = states[k][species];
        }
        return out;
    }
    [[nodiscard]] array<idx> indices_at(view<const real> observation_times) const {
        array<idx> out;
        idx k = 0;
        for (real t : observation_times) {
            while (k + 1 < times.size() && times[k + 1] <= t) {
                ++k;
            }
            out.push_back(k);
        }
        return out;
    }
};

struct leap_options {
    real step = 0.0;     // a fixed leap; zero chooses each leap from epsilon
    real epsilon = 0.03; // expected number of jumps per leap
    real min_step = 1e-6;
};

// many paths of one network, run on the device at once (mk_ssa_run)
struct ssa_ensemble {
    idx paths = 0, species = 0;
    array<int> final_states;      // paths x species
    array<int> observed;          // paths x observation times x species
    array<std::int64_t> steps;    // jumps (Gillespie) or leaps per path
    array<int> bounds;            // the propensity box used
    array<real> observation_times;
    array<trajectory> paths_kept; // with record > 0: each path as the reference returns it
    // mean state at each observation time
    [[nodiscard]] array<vec<real>> means() const {
        const idx n = observation_times.size();
        array<vec<real>> out(n, vec<real>(species, 0.0));
        for (idx p = 0; p < paths; ++p) {
            for (idx k = 0; k < n; ++k) {
                for (idx s = 0; s < species; ++s) {
                    out[k][s] += observed[(p * n + k) * species + s];
                }
            }
        }
        for (auto &m : out) {
            for (real &v : m) {
                v /= static_cast<real>(paths);
            }
        }
        return out;
    }
};

namespace detail {

// mk_ssa_run over a box that doubles until no path leaves it (path i depends on (seed, i)
// alone, so every rerun replays the same paths)
inline ssa_ensemble simulate(const reaction_network &model, const state &initial, real final_time,
                             idx paths, std::uint64_t seed, int method, std::int64_t max_jumps,
                             const leap_options &leap, const array<real> &obs, int record) {
    const idx S = initial.size();
    array<int> bounds(S);
    for (idx s = 0; s < S; ++s) {
        bounds[s] = std::max(2 * initial[s], initial[s] + 64);
    }
    for (;;) {
        const fsp_tables t = tabulate(model, initial, bounds);
        mk_ssa_problem q{};
        mk_ssa_problem_default(&q);
        q.n_species = static_cast<int>(S);
        q.n_reactions = static_cast<int>(model.reactions.size());
        q.bounds = t.bounds.data();
        q.change = t.change.data();
        q.rates = t.rates.data();
        q.initial = t.initial.data();
        q.final_time = final_time;
        q.method = method;
        q.max_jumps = max_jumps;
        q.leap_step = leap.step;
        q.leap_epsilon = leap.epsilon;
        q.leap_min_step = leap.min_step;
        q.paths = static_cast<int64_t>(paths);
        q.seed = seed;
        q.n_observations = static_cast<int>(obs.size());
        q.observation_times = obs.data();
        q.record = record;
        ssa_ensemble e;
        e.paths = paths;
        e.species = S;
        e.bounds = bounds;
        e.observation_times = obs;
        e.final_states.resize(paths * S);
        e.observed.resize(paths * obs.size() * S);
        e.steps.resize(paths);
        array<int> status(paths), rec_states(paths * static_cast<idx>(record) * S), rec_n(record ? paths : 0);
        array<real> rec_times(paths * static_cast<idx>(record));
        mk_ssa_output out{e.final_states.data(), obs.empty() ? nullptr : e.observed.data(),
                          e.steps.data(),        status.data(),
                          record ? rec_times.data() : nullptr,
                          record ? rec_states.data() : nullptr,
                          record ? rec_n.data() : nullptr};
        const int rc = mk_ssa_run(&q, &out, nullptr);
        if (rc == MK_EOVERFLOW) {
            idx size = 1;
            for (int &b : bounds) {
                b = 2 * b + 1;
                size *= static_cast<idx>(b) + 1;
            }
            if (size > (idx(1) << 26)) {
                throw std::overflow_error("ssa: the paths leave every propensity box of at most 2^26 states");
            }
            continue;
        }
        check(rc);
        for (idx p = 0; p < (record ? paths : 0); ++p) {
            const idx n = static_cast<idx>(rec_n[p]);
            if (n > static_cast<idx>(record)) {
                e.paths_kept.push_back({});
                continue;
            }
            trajectory tr;
            for (idx k = 0; k < n; ++k) {
                tr.times.push_back(rec_times[p * record + k]);
                const int *x = rec_states.data() + (p * record + k) * S;
                tr.states.emplace_back(x, x + S);
            }
            e.paths_kept.push_back(std::move(tr));
        }
        return e;
    }
}

template <std::uniform_random_bit_generator Rng>
std::uint64_t seed_from(Rng &random) {
    std::uint64_t s = 0;
    for (int k = 0; k < 4; ++k) {
        s = (s << 16) ^ static_cast<std::uint64_t>(random());
    }
    return s;
}

inline trajectory single_path(const reaction_network &model, const state &x, real final_time,
                              std::uint64_t seed, int method, std::int64_t max_jumps,
                              const leap_options &leap) {
    for (int record = 1024;;) {
        auto e = simulate(model, x, final_time, 1, seed, method, max_jumps, leap, {}, record);
        if (!e.paths_kept.front().states.empty()) {
            return std::move(e.paths_kept.front());
        }
        record *= 4;
    }
}

} // namespace detail

// `paths` independent paths in one device launch: Gillespie (method 0) or tau-leaping (1),
// with the states at the observation times (sorted, within [0, final_time])
inline ssa_ensemble simulate_paths(const reaction_network &model, const state &initial, real final_time,
                                   idx paths, std::uint64_t seed, int method = 0,
                                   array<real> observation_times = {},
                                   std::int64_t max_jumps = std::numeric_limits<std::int64_t>::max(),
                                   const leap_options &leap = {}) {
    return detail::simulate(model, initial, final_time, paths, seed, method, max_jumps, leap,
                            observation_times, 0);
}

// Gillespie's direct method (ssa.hpp:42-74) on the device; `random` seeds the path's stream
template <std::uniform_random_bit_generator Rng>
trajectory gillespie(const reaction_network &model, state x, real final_time, Rng &random,
                     idx max_jumps = std::numeric_limits<idx>::max()) {
    const auto cap = max_jumps > static_cast<idx>(std::numeric_limits<std::int64_t>::max())
                         ? std::numeric_limits<std::int64_t>::max()
                         : static_cast<std::int64_t>(max_jumps);
    return detail::single_path(model, x, final_time, detail::seed_from(random), 0, cap, {});
}

// Poisson tau-leaping (ssa.hpp:83-111) on the device
template <std::uniform_random_bit_generator Rng>
trajectory tau_leaping(const reaction_network &model, state x, real final_time, Rng &random,
                       leap_options options = {}) {
    return detail::single_path(model, x, final_time, detail::seed_from(random), 1,
                               std::numeric_limits<std::int64_t>::max(), options);
}

namespace detail {

// an RDME model as a reaction network over its voxel-major counts: one reaction per (voxel, edge,
// species) hop at n * jump_rate and one per (voxel, local reaction), in the order of
// reaction_diffusion::transitions; the device paths hold at most four counts
template <typename Graph>
reaction_network as_network(const reaction_diffusion<Graph> &m) {
    const idx V = m.n_voxels(), S = m.n_species(), N = V * S;
    if (N > 4) {
        throw std::invalid_argument("ssa: the device paths hold at most four counts; this model has " +
                                    std::to_string(N) + " (voxels x species)");
    }
    reaction_network net;
    for (idx v = 0; v < V; ++v) {
        for (const auto &edge : m.domain.graph.neighbors(v)) {
            for (idx s = 0; s < S; ++s) {
                state change(N, 0);
                const idx from = v * S + s, to = static_cast<idx>(edge.to) * S + s;
                --change[from];
                ++change[to];
                const real hop = m.domain.jump_rate(s, v, edge);
                net.reactions.push_back({change, [from, hop](const state &x) { return x[from] * hop; }});
            }
        }
    }
    for (idx v = 0; v < V; ++v) {
        for (const local_reaction &r : m.reactions) {
            state change(N, 0);
            for (idx s = 0; s < S; ++s) {
                change[v * S + s] = r.change[s];
            }
            const real volume = m.domain.volumes[v];
            const auto rate = r.rate;
            net.reactions.push_back({change, [v, S, volume, rate](const state &x) {
                                         return rate(view<const int>(x.data() + v * S, S), volume);
                                     }});
        }
    }
    return net;
}

} // namespace detail

// Gillespie's direct method on an RDME model (ssa.hpp:42-74 over reaction_diffusion, a
// markov_model): the device paths of its reaction-network form
template <typename Graph, std::uniform_random_bit_generator Rng>
trajectory gillespie(const reaction_diffusion<Graph> &model, state x, real final_time, Rng &random,
                     idx max_jumps = std::numeric_limits<idx>::max()) {
    return gillespie(detail::as_network(model), std::move(x), final_time, random, max_jumps);
}

template <typename Graph, std::uniform_random_bit_generator Rng>
trajectory tau_leaping(const reaction_diffusion<Graph> &model, state x, real final_time, Rng &random,
                       leap_options options = {}) {
    return tau_leaping(detail::as_network(model), std::move(x), final_time, random, options);
}

} // namespace markovkit
