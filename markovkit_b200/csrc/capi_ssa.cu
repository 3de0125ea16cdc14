// C ABI of the batched SSA (ssa.cuh): argument checks, device buffers, one launch, copies out.
#include "capi_internal.hpp"
#include "ssa.cuh"

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

using namespace mkb;
using mkb::capi::as_stream;
using mkb::capi::fail;
using mkb::capi::guarded;

void mk_ssa_problem_default(mk_ssa_problem *p) {
    if (!p) {
        return;
    }
    *p = mk_ssa_problem{};
    p->max_jumps = INT64_MAX;
    p->leap_epsilon = 0.03;
    p->leap_min_step = 1e-6;
    p->paths = 1;
}

int mk_ssa_run(const mk_ssa_problem *problem, mk_ssa_output *out, void *stream) {
    int escaped = 0, capped = 0;
    const int rc = guarded([&] {
        MK_REQUIRE(problem && out, "null argument");
        const mk_ssa_problem &q = *problem;
        MK_REQUIRE(q.n_species >= 1 && q.n_species <= kSsaMaxSpecies, "ssa: 1..4 species");
        MK_REQUIRE(q.n_reactions >= 0 && q.n_reactions <= kSsaMaxReactions, "ssa: 0..16 reactions");
        MK_REQUIRE(q.bounds && q.initial && (q.n_reactions == 0 || (q.change && q.rates)),
                   "ssa: null model arrays");
        MK_REQUIRE(q.method == 0 || q.method == 1, "ssa: method is 0 (Gillespie) or 1 (tau-leaping)");
        MK_REQUIRE(std::isfinite(q.final_time) && q.final_time >= 0.0, "ssa: final_time must be finite and >= 0");
        MK_REQUIRE(q.paths >= 0, "ssa: paths must be >= 0");
        MK_REQUIRE(q.max_jumps >= 0, "ssa: max_jumps must be >= 0");
        MK_REQUIRE(q.method == 0 || (q.leap_step >= 0.0 && q.leap_epsilon > 0.0 && q.leap_min_step > 0.0),
                   "ssa: leap options must be positive");
        MK_REQUIRE(q.n_observations >= 0 && (q.n_observations == 0 || q.observation_times),
                   "ssa: null observation times");
        MK_REQUIRE(q.record >= 0, "ssa: record must be >= 0");
        MK_REQUIRE(out->final_state && out->steps && out->status, "ssa: null outputs");
        MK_REQUIRE(q.n_observations == 0 || out->observed, "ssa: null observation output");
        MK_REQUIRE(q.record == 0 || (out->record_times && out->record_states && out->record_count),
                   "ssa: null trajectory outputs");
        SsaParams p;
        p.S = q.n_species;
        p.R = q.n_reactions;
        std::int64_t box = 1;
        for (int s = q.n_species - 1; s >= 0; --s) {
            MK_REQUIRE(q.bounds[s] >= 0 && q.initial[s] >= 0 && q.initial[s] <= q.bounds[s],
                       "ssa: the initial state must lie in the box");
            p.bounds[s] = q.bounds[s];
            p.initial[s] = q.initial[s];
            p.stride[s] = static_cast<int>(box);
            box *= static_cast<std::int64_t>(q.bounds[s]) + 1;
            MK_REQUIRE(box <= (std::int64_t(1) << 30), "ssa: the propensity box is too large");
        }
        for (int r = 0; r < q.n_reactions; ++r) {
            for (int s = 0; s < q.n_species; ++s) {
                p.change[r][s] = q.change[r * q.n_species + s];
            }
        }
        double prev = 0.0;
        for (int k = 0; k < q.n_observations; ++k) {
            const double t = q.observation_times[k];
            MK_REQUIRE(std::isfinite(t) && t >= prev && t <= q.final_time,
                       "ssa: observation times must be sorted and within [0, final_time]");
            prev = t;
        }
        p.box_size = box;
        p.final_time = q.final_time;
        p.method = q.method;
        p.max_jumps = q.max_jumps;
        p.leap_step = q.leap_step;
        p.leap_epsilon = q.leap_epsilon;
        p.leap_min_step = q.leap_min_step;
        p.paths = q.paths;
        p.seed = q.seed;
        p.n_obs = q.n_observations;
        p.record = q.record;
        if (q.paths == 0) {
            return;
        }
        cudaStream_t st = as_stream(stream);
        const std::int64_t S = q.n_species, P = q.paths;
        std::vector<double> rates(static_cast<std::size_t>(q.n_reactions) * box);
        for (std::size_t i = 0; i < rates.size(); ++i) {
            rates[i] = q.rates[i];
        }
        DeviceArray<double> d_rates, d_obs_t, d_rec_t;
        d_rates.upload(rates.empty() ? std::vector<double>{0.0} : rates);
        d_obs_t.upload(std::vector<double>(q.observation_times, q.observation_times + q.n_observations));
        DeviceArray<int> d_final(static_cast<std::size_t>(P * S)), d_status(static_cast<std::size_t>(P));
        DeviceArray<int> d_obs(static_cast<std::size_t>(P * q.n_observations * S));
        DeviceArray<std::int64_t> d_steps(static_cast<std::size_t>(P));
        DeviceArray<int> d_rec_s, d_rec_n;
        if (q.record > 0) {
            d_rec_t.resize(static_cast<std::size_t>(P * q.record));
            d_rec_s.resize(static_cast<std::size_t>(P * q.record * S));
            d_rec_n.resize(static_cast<std::size_t>(P));
        }
        p.rates = d_rates.get();
        p.obs_times = d_obs_t.get();
        p.final_state = d_final.get();
        p.observed = d_obs.get();
        p.jumps = d_steps.get();
        p.status = d_status.get();
        p.rec_times = d_rec_t.get();
        p.rec_states = d_rec_s.get();
        p.rec_count = d_rec_n.get();
        check_cuda(launch_ssa(p, st), "ssa launch");
        auto copy = [&](void *dst, const void *src, std::size_t bytes) {
            if (bytes) {
                check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "d2h");
            }
        };
        copy(out->final_state, d_final.get(), P * S * sizeof(int));
        copy(out->steps, d_steps.get(), P * sizeof(std::int64_t));
        copy(out->status, d_status.get(), P * sizeof(int));
        if (q.n_observations > 0) {
            copy(out->observed, d_obs.get(), P * q.n_observations * S * sizeof(int));
        }
        if (q.record > 0) {
            copy(out->record_times, d_rec_t.get(), P * q.record * sizeof(double));
            copy(out->record_states, d_rec_s.get(), P * q.record * S * sizeof(int));
            copy(out->record_count, d_rec_n.get(), P * sizeof(int));
        }
        check_cuda(cudaStreamSynchronize(st), "sync");
        for (std::int64_t i = 0; i < P; ++i) {
            escaped += out->status[i] == kEOverflow ? 1 : 0;
            capped += out->status[i] == kENotConv ? 1 : 0;
        }
    });
    if (rc != MK_OK) {
        return rc;
    }
    if (escaped) {
        return fail(MK_EOVERFLOW, "ssa: " + std::to_string(escaped) +
                                      " path(s) left the tabulated box (widen bounds and run again)");
    }
    if (capped) {
        return fail(MK_ENOTCONV, "ssa: " + std::to_string(capped) + " path(s) reached the step cap");
    }
    return MK_OK;
}
