// A MarkovKit-style program against the C++20 facade (include/mk/markovkit.hpp): the calls a
// reference caller makes (population_box, reaction_diffusion, generator, shifted_generator,
// sector_multigrid, num::gmres, solve_krylov_fsp), with checks of the answers. Built by
// tests/test_facade.py; run on a GPU it prints "facade: N checks passed" or exits 1.
#include "mk/markovkit.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>

using namespace markovkit;

namespace {

int checks = 0, failures = 0;

void expect(bool ok, const char *what) {
    ++checks;
    if (!ok) {
        ++failures;
        std::printf("FAILED: %s\n", what);
    }
}

array<local_reaction> birth_death(real birth, real death) {
    return {{{1}, [=](view<const int>, real volume) { return birth * volume; }},
            {{-1}, [=](view<const int> n, real) { return death * n[0]; }}};
}

real norm(const vec<real> &v) { return std::sqrt(std::inner_product(v.begin(), v.end(), v.begin(), 0.0)); }

void spaces() {
    population_box box(16, {3});
    expect(box.size() == 969, "population_box(16, {3}) has 969 states");
    expect(box.n_sectors() == 4 && box.sector_begin(3) == 153, "sector offsets 0/1/17/153");
    for (idx i : {idx(0), idx(5), idx(200), idx(968)}) {
        const auto found = box.find(box[i]);
        expect(found && *found == i, "find(box[i]) == i");
    }
    state outside(16, 0);
    outside[0] = 4;
    expect(!box.find(outside), "a state outside the box is absent");
    population_sector sector(8, {2});
    expect(sector.size() == 36, "population_sector(8, {2}) has C(9, 2) = 36 states");
}

void resolvent() {
    const reaction_diffusion<grid<1>> model{voxel_domain(grid<1>({16}, {1.0 / 16}), {1.0}),
                                      birth_death(0.05, 0.02)};
    population_box box(16, {3});
    const generator Q(box, model, boundary::absorbing);
    constexpr real shift = 0.5;
    const shifted_generator A(Q, shift);
    static_assert(num::linear_operator<shifted_generator, vec<real>, vec<real>>);
    vec<real> b(Q.rows());
    for (idx i = 0; i < b.size(); ++i) {
        b[i] = 1.0 + 0.25 * std::sin(0.37 * static_cast<real>(i));
    }
    // y = s x - Q x by both entry points
    vec<real> qx, ax;
    Q.apply(b, qx);
    A.apply(b, ax);
    real dev = 0.0;
    for (idx i = 0; i < b.size(); ++i) {
        dev = std::max(dev, std::abs(ax[i] - (shift * b[i] - qx[i])));
    }
    expect(dev < 1e-12, "apply_shifted = s x - apply");
    // the assembled operators reproduce the matrix-free ones (tests/test_rdme.cpp:100-158)
    vec<real> mq, ma;
    Q.matrix().apply(b, mq);
    A.matrix().apply(b, ma);
    real dq = 0.0, da = 0.0, sq = 0.0, sa = 0.0;
    for (idx i = 0; i < b.size(); ++i) {
        dq = std::max(dq, std::abs(mq[i] - qx[i]));
        da = std::max(da, std::abs(ma[i] - ax[i]));
        sq = std::max(sq, std::abs(qx[i]));
        sa = std::max(sa, std::abs(ax[i]));
    }
    expect(dq <= 1e-13 * sq && da <= 1e-13 * sa, "matrix().apply = apply (1e-13 relative)");
    expect(Q.matrix().nonzeros() == Q.rows() + Q.n_jumps(), "one entry per jump plus the diagonal");
    const auto exits = Q.exit_rates();
    expect(std::abs(exits[0] - 0.05 * 16 * (1.0 / 16)) < 1e-14, "exit rate of the empty state is the total birth rate");

    const sector_multigrid M(model.domain, box, shift);
    const num::gmres_options options{.tolerance = 1e-10 * norm(b), .max_iterations = 1000, .restart = 30};
    vec<real> x_mg(Q.rows(), 0.0), x_plain(Q.rows(), 0.0), x32(Q.rows(), 0.0);
    const auto mg = num::gmres(A, M, b, x_mg, options);
    // unpreconditioned GMRES(30) stalls on this system; a full Krylov space does not
    const auto plain = num::gmres(A, b, x_plain, {.tolerance = options.tolerance, .max_iterations = 2000, .restart = Q.rows()});
    expect(mg.converged && plain.converged, "both solves converge");
    expect(mg.iterations < plain.iterations, "the multigrid preconditioner cuts iterations");
    vec<real> r;
    A.apply(x_mg, r);
    for (idx i = 0; i < r.size(); ++i) {
        r[i] = b[i] - r[i];
    }
    expect(norm(r) <= 1e-10 * norm(b) * 1.0001, "true residual below 1e-10 relative");
    real diff = 0.0;
    for (idx i = 0; i < b.size(); ++i) {
        diff = std::max(diff, std::abs(x_mg[i] - x_plain[i]));
    }
    expect(diff < 1e-8, "preconditioned and plain solutions agree");
    multigrid_options o32;
    o32.precision = 1;
    const sector_multigrid M32(model.domain, box, shift, o32);
    const auto s32 = num::gmres(A, M32, b, x32, options);
    real d32 = 0.0;
    for (idx i = 0; i < b.size(); ++i) {
        d32 = std::max(d32, std::abs(x32[i] - x_mg[i]));
    }
    expect(s32.converged && d32 < 1e-8 * norm(x_mg), "FP32 multigrid in flexible GMRES agrees");
}

// the reference's benchmark flow (examples/rdme_multigrid_benchmark.cpp:72-121): plain, Jacobi,
// ILU(0) and multigrid preconditioners through one generic num::gmres, and a host operator
template <std::size_t D>
void preconditioners() {
    num::static_array<num::idx, D> dims{};
    dims.fill(4);
    num::static_array<double, D> spacing{};
    spacing.fill(0.25);
    const reaction_diffusion model{voxel_domain(grid<D>(dims, spacing), {4.0}), birth_death(0.05, 0.02)};
    const population_box box(model.n_voxels(), {2});
    const generator Q(box, model, boundary::absorbing);
    constexpr real shift = 0.5;
    const shifted_generator system(Q, shift);
    vec<real> rhs(Q.rows());
    for (idx i = 0; i < rhs.size(); ++i) {
        rhs[i] = 1.0 + 0.1 * std::cos(static_cast<double>(i));
    }
    const num::gmres_options options{.tolerance = 1e-10 * norm(rhs), .max_iterations = 2000,
                                     .restart = std::min<idx>(50, Q.rows())};
    vec<real> inverse_diagonal(Q.rows());
    for (idx i = 0; i < Q.rows(); ++i) {
        inverse_diagonal[i] = 1.0 / (shift + Q.exit_rates()[i]);
    }
    const num::jacobi_preconditioner jacobi(inverse_diagonal);
    const num::ilu0_preconditioner ilu(system.matrix());
    const sector_multigrid<D> mg(model.domain, box, shift);
    expect(mg.max_levels() >= 2, "sector_multigrid<D> builds a hierarchy");
    // any operator with rows(), cols() and apply(x, y) preconditions too (applied on the host)
    struct diagonal_scaling {
        const vec<real> *d;
        [[nodiscard]] idx rows() const { return d->size(); }
        [[nodiscard]] idx cols() const { return d->size(); }
        void apply(const vec<real> &x, vec<real> &y) const {
            y.resize(x.size());
            for (idx i = 0; i < x.size(); ++i) {
                y[i] = (*d)[i] * x[i];
            }
        }
    } host{&inverse_diagonal};
    vec<real> xp(Q.rows(), 0.0), xj(Q.rows(), 0.0), xi(Q.rows(), 0.0), xm(Q.rows(), 0.0), xh(Q.rows(), 0.0);
    const auto rp = num::gmres(system, rhs, xp, options);
    const auto rj = num::gmres(system, jacobi, rhs, xj, options);
    const auto ri = num::gmres(system, ilu, rhs, xi, options);
    const auto rm = num::gmres(system, mg, rhs, xm, options);
    const auto rh = num::gmres(system, host, rhs, xh, options);
    expect(rp.converged && rj.converged && ri.converged && rm.converged && rh.converged,
           "plain, jacobi, ilu0, multigrid and host-operator GMRES converge");
    expect(ri.iterations < rj.iterations, "ILU(0) takes fewer iterations than Jacobi");
    expect(rh.iterations == rj.iterations && xh == xj, "a host d .* v gives the Jacobi iterates");
    real diff = 0.0, scale = 0.0;
    for (idx i = 0; i < Q.rows(); ++i) {
        diff = std::max({diff, std::abs(xj[i] - xm[i]), std::abs(xi[i] - xm[i]), std::abs(xp[i] - xm[i])});
        scale = std::max(scale, std::abs(xm[i]));
    }
    expect(diff <= 1e-8 * scale, "every preconditioner reaches the same solution");
    // generator::jumps(j): in-space jumps plus the leak make up the exit rate
    real worst = 0.0;
    idx total = 0;
    for (idx j = 0; j < Q.rows(); ++j) {
        real out = Q.leak_rates()[j];
        for (const auto &e : Q.jumps(j)) {
            out += e.rate;
            ++total;
        }
        worst = std::max(worst, std::abs(out - Q.exit_rates()[j]) / std::max(Q.exit_rates()[j], 1.0));
    }
    expect(worst < 1e-14 && total == Q.n_jumps(), "jumps(j) and leak_rates() add up to exit_rates()");
}

void annihilation_transform() {
    // A + B -> nothing at rate 2 a b / V; E[exp(-sT)] + s S_hat(s) = 1 for the annihilation time
    const reaction_diffusion<grid<1>> model{
        voxel_domain(grid<1>({4}, {0.25}), {1.0, 1.0}),
        {{{-1, -1}, [](view<const int> n, real volume) { return 2.0 * n[0] * n[1] / volume; }}}};
    population_box box(4, {1, 1});
    const generator Q(box, model);
    expect(Q.rows() == 25, "1 + V + V + V^2 states");
    constexpr real shift = 0.5;
    const shifted_generator A(Q, shift);
    const sector_multigrid M(model.domain, box, shift);
    const idx joint = *box.find_sector({1, 1});
    const idx vacuum = *box.find(state(8, 0));
    state initial(8, 0);
    initial[model.index(0, 0)] = 1;
    initial[model.index(2, 1)] = 1;
    vec<real> b(Q.rows(), 0.0), x(Q.rows(), 0.0);
    b[*box.find(initial)] = 1.0;
    const auto res = num::gmres(A, M, b, x, {.tolerance = 1e-12, .max_iterations = 200, .restart = 25});
    expect(res.converged, "transform solve converges");
    real survival = 0.0;
    for (idx i = box.sector_begin(joint); i < box.sector_end(joint); ++i) {
        survival += x[i];
    }
    expect(std::abs(shift * x[vacuum] + shift * survival - 1.0) < 1e-10, "E[exp(-sT)] + s S(s) = 1");
}

void krylov_fsp() {
    const reaction_network death{{{{-1}, [](const state &x) { return real(x[0]); }}}};
    krylov_fsp_options o;
    o.inside = box({5});
    o.tolerance = 1e-10;
    o.max_steps = 100;
    o.krylov_tol = 1e-12;
    const auto sol = solve_krylov_fsp(death, {5}, 1.0, o);
    expect(sol.times.back() == 1.0, "Krylov FSP reaches the final time");
    const auto m = sol.means();
    expect(m.rows() == 2 && std::abs(m(1, 0) - 5.0 * std::exp(-1.0)) < 1e-8, "pure-death mean");
    expect(std::abs(sol.snapshots.back().marginal(0).at(0) - std::pow(1.0 - std::exp(-1.0), 5)) < 1e-8,
           "extinction probability");
}

// the reference's adaptive test (tests/test_fsp.cpp:68-77), written as the reference writes it
void adaptive_fsp() {
    const reaction_network birth_death{{{{1}, [](const state &) { return 5.0; }},
                                        {{-1}, [](const state &x) { return 0.1 * x[0]; }}}};
    const auto solution = solve_adaptive_fsp(birth_death, {0}, 2.0, {.inside = box({100}), .step_scale = 0.1});
    expect(solution.times.size() > 1, "adaptive FSP saves snapshots");
    const real exact = (5.0 / 0.1) * (1.0 - std::exp(-0.1 * 2.0));
    const auto m = solution.means();
    expect(std::abs(m(m.rows() - 1, 0) - exact) < 0.1, "adaptive FSP matches the birth-death mean");
}

// everywhere() (the default region): the device box grows until no expansion meets it, and the
// result is the one of a box the support never reaches
void fsp_everywhere() {
    const reaction_network birth_death{{{{1}, [](const state &) { return 5.0; }},
                                        {{-1}, [](const state &x) { return 0.1 * x[0]; }}}};
    krylov_fsp_options o;
    o.tolerance = 1e-8;
    const auto grown = solve_krylov_fsp(birth_death, {0}, 2.0, o);
    o.inside = box(400);
    const auto boxed = solve_krylov_fsp(birth_death, {0}, 2.0, o);
    const distribution &a = grown.snapshots.back(), &b = boxed.snapshots.back();
    expect(a.size() == b.size() && a.size() > 17, "everywhere() grows past the first box");
    real diff = 0.0;
    for (idx i = 0; i < a.size() && i < b.size(); ++i) {
        expect(a[i] == b[i], "the same support in the same order");
        diff = std::max(diff, std::abs(a.probabilities()[i] - b.probabilities()[i]));
    }
    expect(diff <= 1e-14, "everywhere() matches a box the support never reaches");
    const real exact = (5.0 / 0.1) * (1.0 - std::exp(-0.1 * 2.0));
    expect(std::abs(grown.means()(1, 0) - exact) < 1e-6, "the birth-death mean");

    // a listed generator over a support built on the host (generator.hpp:27-44)
    distribution p(state{0});
    expand(p, birth_death, box(10), 3);
    expect(p.size() == 4, "three rings from {0}");
    const generator Q(p, birth_death, boundary::reflecting);
    vec<real> x{0.1, 0.2, 0.3, 0.4}, y, z;
    Q.apply(x, y);
    Q.matrix().apply(x, z);
    real sum = 0.0;
    for (idx i = 0; i < 4; ++i) {
        expect(std::abs(y[i] - z[i]) < 1e-15, "device apply equals the assembled matrix");
        sum += y[i];
    }
    expect(std::abs(sum) < 1e-15, "a reflecting generator conserves probability");
    expect(Q.leak_rates()[3] == 5.0 && std::abs(Q.exit_rates()[3] - 0.3) < 1e-15, "the birth out of {3} leaks");
}

} // namespace

int main() {
    try {
        spaces();
        resolvent();
        preconditioners<1>();
        preconditioners<2>();
        preconditioners<3>();
        annihilation_transform();
        krylov_fsp();
        adaptive_fsp();
        fsp_everywhere();
    } catch (const std::exception &e) {
        std::printf("FAILED with exception: %s\n", e.what());
        return 1;
    }
    if (failures) {
        std::printf("facade: %d of %d checks failed\n", failures, checks);
        return 1;
    }
    std::printf("facade: %d checks passed\n", checks);
    return 0;
}
