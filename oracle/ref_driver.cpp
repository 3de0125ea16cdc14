// ORACLE TEST INFRASTRUCTURE — runs the reference's own resolvent path on one seeded problem.
//
// Compiled by oracle/Makefile from MarkovKit's headers where they lie (include/markovkit/**)
// against the project-written numerics shim; outputs go to a directory given on the command
// line. The problem families restate the reference's own models: birth-death in every voxel
// (tests/test_rdme.cpp:16-20, README "An RDME..."), A + B -> 0 annihilation
// (examples/rdme_two_particle_annihilation.cpp:61-65) and pure diffusion. The call sequence is
// the reference's (README; examples/rdme_multigrid_benchmark.cpp:72-121):
//   population_box -> generator -> shifted_generator -> sector_multigrid -> num::gmres.
//
// usage: ref_driver key=value ...   (see parse() below for the keys)
#include "markovkit.hpp"
#include "linear/solvers/gmres.hpp"
#include "seeded.hpp"
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>

using namespace markovkit;

namespace {

using clock_type = std::chrono::steady_clock;

double ms_since(clock_type::time_point t0) {
    return std::chrono::duration<double, std::milli>(clock_type::now() - t0).count();
}

struct args {
    std::map<std::string, std::string> kv;
    std::string get(const std::string &k, const std::string &d) const {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
    double num(const std::string &k, double d) const {
        auto it = kv.find(k);
        return it == kv.end() ? d : std::stod(it->second);
    }
    long integer(const std::string &k, long d) const {
        auto it = kv.find(k);
        return it == kv.end() ? d : std::stol(it->second);
    }
};

std::vector<double> list_of(const std::string &s) {
    std::vector<double> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) {
        out.push_back(std::stod(item));
    }
    return out;
}

void write_f64(const std::string &path, const std::vector<double> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), static_cast<std::streamsize>(v.size() * 8));
}

std::vector<double> read_f64(const std::string &path, std::size_t n) {
    std::vector<double> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(n * 8));
    if (!f) {
        throw std::runtime_error("short read: " + path);
    }
    return v;
}

std::string json_list(const std::vector<double> &v) {
    std::ostringstream o;
    o.precision(17);
    o << '[';
    for (std::size_t i = 0; i < v.size(); ++i) {
        o << (i ? "," : "") << v[i];
    }
    o << ']';
    return o.str();
}

template <std::size_t D>
int run(const args &a) {
    const idx cells = static_cast<idx>(a.integer("cells", 16));
    const double h = a.num("h", 1.0 / static_cast<double>(cells));
    num::static_array<idx, D> dims{};
    dims.fill(cells);
    num::static_array<double, D> spacing{};
    spacing.fill(h);
    const std::string family = a.get("model", "birth_death");
    const double birth = a.num("birth", 0.05), death = a.num("death", 0.02);
    const double k_react = a.num("k", 10.0);

    array<real> diffusivities;
    array<local_reaction> reactions;
    if (family == "birth_death") {
        diffusivities = {a.num("D", 1.0)};
        reactions = {{{1}, [=](view<const int>, real volume) { return birth * volume; }},
                     {{-1}, [=](view<const int> n, real) { return death * n[0]; }}};
    } else if (family == "annihilation") {
        diffusivities = {a.num("D", 1.0), a.num("D2", a.num("D", 1.0))};
        reactions = {{{-1, -1}, [=](view<const int> n, real volume) {
                          return k_react * n[0] * n[1] / volume;
                      }}};
    } else if (family == "diffusion") {
        diffusivities = {a.num("D", 1.0)};
    } else {
        throw std::invalid_argument("unknown model " + family);
    }
    const reaction_diffusion<grid<D>> model{
        voxel_domain(grid<D>(dims, spacing), diffusivities), reactions};

    array<int> caps;
    for (double c : list_of(a.get("cap", "3"))) {
        caps.push_back(static_cast<int>(c));
    }
    if (caps.size() != model.n_species()) {
        throw std::invalid_argument("one cap per species");
    }
    const boundary leaks =
        a.get("boundary", "absorbing") == "reflecting" ? boundary::reflecting : boundary::absorbing;
    const real shift = a.num("shift", 0.5);
    const std::string out = a.get("out", ".");

    auto t0 = clock_type::now();
    const population_box box(model.n_voxels(), caps);
    const double box_ms = ms_since(t0);
    t0 = clock_type::now();
    const generator Q(box, model, leaks);
    const double gen_ms = ms_since(t0);
    const idx N = Q.rows();
    const shifted_generator A(Q, shift);

    std::ostringstream meta;
    meta.precision(17);
    meta << "{\"N\":" << N << ",\"n_jumps\":" << Q.n_jumps() << ",\"n_sectors\":"
         << box.n_sectors() << ",\"box_ms\":" << box_ms << ",\"generator_ms\":" << gen_ms;
    std::vector<double> begins;
    for (idx k = 0; k <= box.n_sectors(); ++k) {
        begins.push_back(static_cast<double>(k < box.n_sectors() ? box.sector_begin(k) : N));
    }
    meta << ",\"sector_begin\":" << json_list(begins);

    if (a.integer("dump_states", 0)) {
        std::ofstream f(out + "/states.i32", std::ios::binary);
        for (idx i = 0; i < N; ++i) {
            f.write(reinterpret_cast<const char *>(box[i].data()),
                    static_cast<std::streamsize>(box[i].size() * 4));
        }
        std::vector<double> found(N);
        for (idx i = 0; i < N; ++i) {
            found[i] = static_cast<double>(*box.find(box[i]));
        }
        write_f64(out + "/find.f64", found);
    }

    if (a.integer("do_apply", 1)) {
        write_f64(out + "/exit.f64", std::vector<double>(Q.exit_rates().begin(), Q.exit_rates().end()));
        write_f64(out + "/leak.f64", std::vector<double>(Q.leak_rates().begin(), Q.leak_rates().end()));
        const std::string xfile = a.get("x_file", "");
        const vec<real> x = xfile.empty() ? oracle::uniform_vector(a.integer("seed", 0) + 1000, N)
                                          : read_f64(xfile, N);
        vec<real> y(N, 0.0), z(N, 0.0);
        Q.apply(x, y);
        A.apply(x, z);
        write_f64(out + "/x.f64", x);
        write_f64(out + "/Qx.f64", y);
        write_f64(out + "/Ax.f64", z);
    }

    // the assembled Q and shift I - Q (generator.hpp:84-107) as CSR: <name>_ptr, _col, _val
    if (a.integer("dump_matrix", 0)) {
        const auto dump = [&](const std::string &name, const num::spmat &m) {
            write_f64(out + "/" + name + "_ptr.f64",
                      std::vector<double>(m.row_ptr().begin(), m.row_ptr().end()));
            write_f64(out + "/" + name + "_col.f64",
                      std::vector<double>(m.columns().begin(), m.columns().end()));
            write_f64(out + "/" + name + "_val.f64",
                      std::vector<double>(m.values().begin(), m.values().end()));
        };
        dump("Qm", Q.matrix());
        dump("Am", A.matrix());
    }

    // generator::jumps(j) for every j in the reference's order (generator.hpp:50-53):
    // jumps_first = offsets (N + 1), jumps_to, jumps_rate
    if (a.integer("dump_jumps", 0)) {
        std::vector<double> first{0.0}, to, rate;
        for (idx j = 0; j < N; ++j) {
            for (const auto &e : Q.jumps(j)) {
                to.push_back(static_cast<double>(e.to));
                rate.push_back(e.rate);
            }
            first.push_back(static_cast<double>(to.size()));
        }
        write_f64(out + "/jumps_first.f64", first);
        write_f64(out + "/jumps_to.f64", to);
        write_f64(out + "/jumps_rate.f64", rate);
    }

    const std::string rhs_kind = a.get("rhs", "uniform");
    const std::uint64_t seed = static_cast<std::uint64_t>(a.integer("seed", 0));
    vec<real> b;
    if (rhs_kind == "uniform") {
        b = oracle::uniform_rhs(seed, N);
    } else if (rhs_kind == "dirichlet") {
        b = oracle::dirichlet_rhs(seed, N);
    } else {
        b = read_f64(rhs_kind, N);
    }
    write_f64(out + "/b.f64", b);

    multigrid_options mgo;
    mgo.pre_sweeps = static_cast<int>(a.integer("pre", 2));
    mgo.post_sweeps = static_cast<int>(a.integer("post", 2));
    mgo.jacobi_weight = a.num("omega", 2.0 / 3.0);
    mgo.coarsest_size = static_cast<idx>(a.integer("coarsest", 4));
    mgo.max_levels = static_cast<int>(a.integer("max_levels", 32));
    mgo.coarse_cycles = static_cast<int>(a.integer("cycles", 1));
    mgo.sweep_growth = static_cast<int>(a.integer("growth", 0));
    if (a.get("smoother", "jacobi") == "aggregate") {
        mgo.smoother = relaxation::aggregate_block;
    }

    if (a.integer("do_mg", 1)) {
        t0 = clock_type::now();
        const sector_multigrid<D> M(model.domain, box, shift, mgo);
        const double mg_ms = ms_since(t0);
        meta << ",\"mg_setup_ms\":" << mg_ms << ",\"mg_levels\":" << M.max_levels();
        vec<real> z(N, 0.0);
        t0 = clock_type::now();
        M.apply(b, z);
        meta << ",\"mg_apply_ms\":" << ms_since(t0);
        write_f64(out + "/Mb.f64", z);

        if (a.integer("do_gmres", 1)) {
            const double rel = a.num("tol", 1e-10);
            double bnorm = 0.0;
            for (double v : b) {
                bnorm += v * v;
            }
            bnorm = std::sqrt(bnorm);
            const num::gmres_options options{
                .tolerance = rel * bnorm,
                .max_iterations = static_cast<idx>(a.integer("maxit", 1000)),
                .restart = static_cast<idx>(a.integer("restart", 30))};
            const long warmup = a.integer("warmup", 0), solves = a.integer("solves", 1);
            // sample_iters > 0: after the warm-up solves, each timed solve stops after this many
            // Arnoldi steps (a bounded sample of a full solve)
            const long sample = a.integer("sample_iters", 0);
            std::vector<double> solve_ms;
            vec<real> x(N, 0.0);
            num::solver_result result, full;
            for (long s = 0; s < warmup + solves; ++s) {
                std::fill(x.begin(), x.end(), 0.0);
                num::gmres_options run = options;
                if (sample > 0 && s >= warmup) {
                    run.max_iterations = static_cast<idx>(sample);
                }
                t0 = clock_type::now();
                result = num::gmres(A, M, b, x, run);
                const double t = ms_since(t0);
                if (s >= warmup) {
                    solve_ms.push_back(t);
                } else {
                    full = result;
                }
            }
            if (warmup > 0) {
                meta << ",\"full_solve_iterations\":" << full.iterations;
            }
            vec<real> r(N, 0.0);
            A.apply(x, r);
            double rn = 0.0;
            for (idx i = 0; i < N; ++i) {
                rn += (b[i] - r[i]) * (b[i] - r[i]);
            }
            write_f64(out + "/x_mg.f64", x);
            meta << ",\"gmres_mg\":{\"iterations\":" << result.iterations
                 << ",\"residual\":" << result.residual << ",\"converged\":" << result.converged
                 << ",\"true_rel_residual\":" << std::sqrt(rn) / bnorm
                 << ",\"solve_ms\":" << json_list(solve_ms) << "}";
        }
    }
    if (a.integer("do_plain", 0)) {
        double bnorm = 0.0;
        for (double v : b) {
            bnorm += v * v;
        }
        bnorm = std::sqrt(bnorm);
        const num::gmres_options options{
            .tolerance = a.num("tol", 1e-10) * bnorm,
            .max_iterations = static_cast<idx>(a.integer("maxit", 1000)),
            .restart = static_cast<idx>(a.integer("restart", 30))};
        vec<real> x(N, 0.0);
        t0 = clock_type::now();
        const auto result = num::gmres(A, b, x, options);
        meta << ",\"gmres_plain\":{\"iterations\":" << result.iterations
             << ",\"residual\":" << result.residual << ",\"converged\":" << result.converged
             << ",\"solve_ms\":" << ms_since(t0) << "}";
        write_f64(out + "/x_plain.f64", x);
    }

    // first-level transfer and coarse operator of every sector's own population_multigrid
    if (a.integer("do_transfer", 0)) {
        meta << ",\"transfer\":[";
        bool first = true;
        for (idx k = 0; k < box.n_sectors(); ++k) {
            const population_multigrid<D> level(model.domain, box.sector_totals(k), shift, mgo);
            if (!level.coarse_level()) {
                continue;
            }
            const idx nf = level.rows(), nc = level.transfer().coarse_size();
            vec<real> c = oracle::uniform_vector(seed + 77 + k, nc), f(nf, 0.0), rc(nc, 0.0);
            const vec<real> g = oracle::uniform_vector(seed + 99 + k, nf);
            level.transfer().prolong(c, f);
            level.transfer().restrict(g, rc);
            vec<real> Af(nf, 0.0), Ac(nc, 0.0);
            level.apply_system(f, Af);
            level.coarse_level()->apply_system(c, Ac);
            const std::string tag = out + "/sector" + std::to_string(k);
            write_f64(tag + "_c.f64", c);
            write_f64(tag + "_Pc.f64", f);
            write_f64(tag + "_g.f64", g);
            write_f64(tag + "_Rg.f64", rc);
            write_f64(tag + "_APc.f64", Af);
            write_f64(tag + "_Acc.f64", Ac);
            vec<real> cyc(nf, 0.0);
            level.apply(g, cyc);
            write_f64(tag + "_cycle_g.f64", cyc);
            meta << (first ? "" : ",") << "{\"sector\":" << k << ",\"fine\":" << nf
                 << ",\"coarse\":" << nc << ",\"levels\":" << level.n_levels() << "}";
            first = false;
        }
        meta << "]";
    }
    meta << "}";
    std::ofstream(out + "/meta.json") << meta.str() << '\n';
    std::cout << meta.str() << '\n';
    return 0;
}

} // namespace

int main(int argc, char **argv) {
    args a;
    for (int i = 1; i < argc; ++i) {
        const std::string s(argv[i]);
        const auto eq = s.find('=');
        if (eq == std::string::npos) {
            std::cerr << "expected key=value, got " << s << '\n';
            return 2;
        }
        a.kv[s.substr(0, eq)] = s.substr(eq + 1);
    }
    try {
        switch (a.integer("dim", 1)) {
        case 1:
            return run<1>(a);
        case 2:
            return run<2>(a);
        case 3:
            return run<3>(a);
        default:
            std::cerr << "dim must be 1, 2 or 3\n";
            return 2;
        }
    } catch (const std::exception &e) {
        std::cerr << "ref_driver: " << e.what() << '\n';
        return 1;
    }
}
