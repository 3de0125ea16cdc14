// ORACLE TEST INFRASTRUCTURE — times the reference's own gillespie / tau_leaping
// (markovkit/ssa.hpp:42-113) on one core, for the CPU baseline of the batched SSA.
//
// Compiled by oracle/Makefile from MarkovKit's headers where they lie, against the numerics
// shim (num::rng = a seeded 64-bit Mersenne twister). The networks restate the toggle switch and
// birth-death models of markovkit_b200/fsp_models.py.
//
// usage: ref_ssa model=toggle|birth_death paths=N T=t seed=s method=gillespie|tau_leaping
//        prints {"paths":..,"seconds":..,"mean":[..]}
#include "markovkit.hpp"
#include "stochastic/rng.hpp"
#include <chrono>
#include <cmath>
#include <cstdio>
#include <map>
#include <string>

using namespace markovkit;

int main(int argc, char **argv) {
    std::map<std::string, std::string> kv;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        const auto eq = a.find('=');
        if (eq != std::string::npos) {
            kv[a.substr(0, eq)] = a.substr(eq + 1);
        }
    }
    auto get = [&](const char *k, const char *d) { return kv.count(k) ? kv[k] : std::string(d); };
    const std::string family = get("model", "toggle");
    const long paths = std::stol(get("paths", "1000"));
    const double T = std::stod(get("T", "2.0"));
    const bool leap = get("method", "gillespie") == "tau_leaping";
    num::rng random(std::stoull(get("seed", "1")));
    reaction_network model;
    state x0;
    if (family == "toggle") {
        const double a1 = std::stod(get("a1", "30")), a2 = std::stod(get("a2", "25"));
        const double n1 = std::stod(get("n1", "2")), n2 = std::stod(get("n2", "2.5"));
        model = reaction_network{{{{1, 0}, [=](const state &x) { return a1 / (1.0 + std::pow(double(x[1]), n1)); }},
                                  {{0, 1}, [=](const state &x) { return a2 / (1.0 + std::pow(double(x[0]), n2)); }},
                                  {{-1, 0}, [](const state &x) { return double(x[0]); }},
                                  {{0, -1}, [](const state &x) { return double(x[1]); }}}};
        x0 = {0, 0};
    } else {
        const double b = std::stod(get("birth", "5")), d = std::stod(get("death", "0.1"));
        model = reaction_network{{{{1}, [=](const state &) { return b; }},
                                  {{-1}, [=](const state &x) { return d * x[0]; }}}};
        x0 = {0};
    }
    std::vector<double> mean(x0.size(), 0.0);
    const auto t0 = std::chrono::steady_clock::now();
    for (long p = 0; p < paths; ++p) {
        const trajectory path = leap ? tau_leaping(model, x0, T, random) : gillespie(model, x0, T, random);
        for (std::size_t s = 0; s < x0.size(); ++s) {
            mean[s] += path.states.back()[s];
        }
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("{\"paths\":%ld,\"seconds\":%.6f,\"mean\":[", paths, sec);
    for (std::size_t s = 0; s < mean.size(); ++s) {
        std::printf("%s%.6f", s ? "," : "", mean[s] / static_cast<double>(paths));
    }
    std::printf("]}\n");
    return 0;
}
