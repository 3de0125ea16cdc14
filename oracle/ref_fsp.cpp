// ORACLE TEST INFRASTRUCTURE — runs the reference's own Krylov FSP (markovkit/fsp.hpp:190-254)
// on reaction networks of the benchmark's two families, compiled from MarkovKit's headers where
// they lie against the project-written numerics shim (oracle/Makefile).
//
// Instances are read one per line from a file (or stdin):
//   birth_death <birth> <death> <bound> <T> <tol> <krylov_tol> <krylov_dim> <x0>
//   toggle <a1> <a2> <n1> <n2> <bound_x> <bound_y> <T> <tol> <krylov_tol> <krylov_dim> <x0> <y0>
//   table <key>=<value> ...
// The birth_death and toggle lines may end in <key>=<value> options as the table line takes.
// adaptive=1 runs solve_adaptive_fsp (fsp.hpp:123-188) instead, with the keys scale, prune, flux
// and minp for adaptive_fsp_options' step_scale, prune_fraction, flux_tolerance, min_probability.
// Birth-death: {+1} at rate birth, {-1} at rate death * x. Toggle switch: {+1,0} at
// a1 / (1 + y^n1), {0,+1} at a2 / (1 + x^n2), unit degradation {-1,0} at x and {0,-1} at y.
// Table: any network whose propensities are tabulated over the box, read from path=<file>
// (int32 S, int32 R, int32 bounds[S], int32 change[R][S], float64 rates[R][box], box index
// with species 0 most significant); keys T, tol, ktol, kdim, layers, step, growth, drop_p,
// drop_d, max_steps and init=<x0,x1,...> set the problem and krylov_fsp_options.
// The region is box(bounds) (fsp.hpp:26-35). For each instance it prints one JSON line with the
// final time, the support and wall time, and writes the final distribution as (box index, p)
// pairs to <out>/fsp<k>.bin when out=<dir> is given (box index: species 0 most significant).
//
// usage: ref_fsp file=<instances> [out=<dir>] [limit=<n>]
#include "markovkit.hpp"

#include <chrono>
#include <cmath>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

using namespace markovkit;

namespace {

// the <key>=<value> tokens left on an instance line
void read_options(std::istringstream &in, std::map<std::string, std::string> &o) {
    std::string tok;
    while (in >> tok) {
        const auto eq = tok.find('=');
        if (eq != std::string::npos) {
            o[tok.substr(0, eq)] = tok.substr(eq + 1);
        }
    }
}

} // namespace

int main(int argc, char **argv) {
    std::map<std::string, std::string> kv;
    for (int i = 1; i < argc; ++i) {
        const std::string s(argv[i]);
        const auto eq = s.find('=');
        if (eq != std::string::npos) {
            kv[s.substr(0, eq)] = s.substr(eq + 1);
        }
    }
    std::ifstream file(kv.count("file") ? kv["file"] : "/dev/stdin");
    const std::string out = kv.count("out") ? kv["out"] : "";
    const long limit = kv.count("limit") ? std::stol(kv["limit"]) : -1;
    std::string line;
    long k = 0;
    while (std::getline(file, line) && (limit < 0 || k < limit)) {
        std::istringstream in(line);
        std::string family;
        in >> family;
        if (family.empty()) {
            continue;
        }
        reaction_network model;
        array<int> bounds;
        state x0;
        double T = 0, tol = 0, ktol = 0;
        int kdim = 30;
        std::map<std::string, std::string> extra;
        if (family == "birth_death") {
            double b, d;
            int bound, x;
            in >> b >> d >> bound >> T >> tol >> ktol >> kdim >> x;
            model.reactions = {{{1}, [=](const state &) { return b; }},
                               {{-1}, [=](const state &s) { return d * s[0]; }}};
            bounds = {bound};
            x0 = {x};
            read_options(in, extra);
        } else if (family == "toggle") {
            double a1, a2, n1, n2;
            int bx, by, x, y;
            in >> a1 >> a2 >> n1 >> n2 >> bx >> by >> T >> tol >> ktol >> kdim >> x >> y;
            model.reactions = {
                {{1, 0}, [=](const state &s) { return a1 / (1.0 + std::pow(double(s[1]), n1)); }},
                {{0, 1}, [=](const state &s) { return a2 / (1.0 + std::pow(double(s[0]), n2)); }},
                {{-1, 0}, [](const state &s) { return double(s[0]); }},
                {{0, -1}, [](const state &s) { return double(s[1]); }}};
            bounds = {bx, by};
            x0 = {x, y};
            read_options(in, extra);
        } else if (family == "table") {
            std::map<std::string, std::string> o;
            std::string tok;
            while (in >> tok) {
                const auto eq = tok.find('=');
                if (eq != std::string::npos) {
                    o[tok.substr(0, eq)] = tok.substr(eq + 1);
                }
            }
            std::ifstream tf(o.at("path"), std::ios::binary);
            std::int32_t S = 0, R = 0;
            tf.read(reinterpret_cast<char *>(&S), 4);
            tf.read(reinterpret_cast<char *>(&R), 4);
            std::vector<std::int32_t> b(S), ch(static_cast<std::size_t>(R) * S);
            tf.read(reinterpret_cast<char *>(b.data()), 4 * S);
            tf.read(reinterpret_cast<char *>(ch.data()), 4 * ch.size());
            std::size_t box_size = 1;
            for (int s = 0; s < S; ++s) {
                box_size *= static_cast<std::size_t>(b[s]) + 1;
            }
            auto rates = std::make_shared<std::vector<double>>(static_cast<std::size_t>(R) * box_size);
            tf.read(reinterpret_cast<char *>(rates->data()), 8 * rates->size());
            if (!tf) {
                std::cerr << "short table file\n";
                return 2;
            }
            bounds.assign(b.begin(), b.end());
            for (int r = 0; r < R; ++r) {
                state change(ch.begin() + static_cast<std::ptrdiff_t>(r) * S,
                             ch.begin() + static_cast<std::ptrdiff_t>(r + 1) * S);
                const std::vector<int> bb(b.begin(), b.end());
                model.reactions.push_back(
                    {change, [=](const state &x) {
                         std::size_t i = 0;
                         for (std::size_t s = 0; s < bb.size(); ++s) {
                             i = i * (bb[s] + 1) + x[s];
                         }
                         return (*rates)[static_cast<std::size_t>(r) * box_size + i];
                     }});
            }
            T = std::stod(o.at("T"));
            tol = o.count("tol") ? std::stod(o["tol"]) : 1e-6;
            ktol = o.count("ktol") ? std::stod(o["ktol"]) : 1e-8;
            kdim = o.count("kdim") ? std::stoi(o["kdim"]) : 30;
            std::stringstream init(o.at("init"));
            std::string c;
            while (std::getline(init, c, ',')) {
                x0.push_back(std::stoi(c));
            }
            extra = o;
        } else {
            std::cerr << "unknown family " << family << '\n';
            return 2;
        }
        krylov_fsp_options opt;
        opt.inside = box(bounds);
        opt.tolerance = tol;
        opt.krylov_tol = ktol;
        opt.krylov_dim = kdim;
        if (extra.count("layers")) {
            opt.layers = std::stoi(extra["layers"]);
        }
        if (extra.count("step")) {
            opt.initial_step = std::stod(extra["step"]);
        }
        if (extra.count("growth")) {
            opt.step_growth = std::stod(extra["growth"]);
        }
        if (extra.count("drop_p")) {
            opt.drop_probability = std::stod(extra["drop_p"]);
        }
        if (extra.count("drop_d")) {
            opt.drop_derivative = std::stod(extra["drop_d"]);
        }
        if (extra.count("max_steps")) {
            opt.max_steps = std::stoi(extra["max_steps"]);
        }
        const auto t0 = std::chrono::steady_clock::now();
        fsp_solution sol;
        if (extra.count("adaptive") && extra["adaptive"] == "1") {
            // solve_adaptive_fsp (fsp.hpp:123-188) with adaptive_fsp_options from the keys
            // scale, prune, flux, minp (and layers, max_steps, kdim, ktol as above)
            adaptive_fsp_options ao;
            ao.inside = box(bounds);
            ao.krylov_dim = kdim;
            ao.krylov_tol = ktol;
            ao.layers = opt.layers;
            ao.max_steps = opt.max_steps;
            if (extra.count("scale")) {
                ao.step_scale = std::stod(extra["scale"]);
            }
            if (extra.count("prune")) {
                ao.prune_fraction = std::stod(extra["prune"]);
            }
            if (extra.count("flux")) {
                ao.flux_tolerance = std::stod(extra["flux"]);
            }
            if (extra.count("minp")) {
                ao.min_probability = std::stod(extra["minp"]);
            }
            sol = solve_adaptive_fsp(model, x0, T, ao);
        } else {
            sol = solve_krylov_fsp(model, x0, T, opt);
        }
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        const distribution &p = sol.snapshots.back();
        if (!out.empty()) {
            std::ofstream f(out + "/fsp" + std::to_string(k) + ".bin", std::ios::binary);
            for (idx i = 0; i < p.size(); ++i) {
                std::int64_t index = 0;
                for (idx s = 0; s < bounds.size(); ++s) {
                    index = index * (bounds[s] + 1) + p[i][s];
                }
                const double prob = p.probabilities()[i];
                f.write(reinterpret_cast<const char *>(&index), 8);
                f.write(reinterpret_cast<const char *>(&prob), 8);
            }
        }
        std::cout.precision(17);
        std::cout << "{\"k\":" << k << ",\"t\":" << sol.times.back() << ",\"support\":" << p.size()
                  << ",\"saved\":" << sol.times.size() << ",\"ms\":" << ms << "}" << std::endl;
        ++k;
    }
    return 0;
}
