// The C ABI of batched Krylov FSP (include/markovkit_b200.h, "Krylov FSP"): checks and packs
// the instances, uploads their propensity tables, sizes the per-block workspace, launches the
// persistent kernel of fsp.cu and picks its block shape by timing.
#include "capi_internal.hpp"
#include "fsp.cuh"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

struct mk_fsp_batch_s {
    int n = 0;
    std::vector<mkb::FspInstance> inst;     // queue order: largest box first
    std::vector<std::int64_t> out_offset;   // by instance
    std::int64_t total_box = 0;
    std::int64_t cap = 0;                   // largest box
    int rmax = 0;                           // most reactions
    mkb::DeviceArray<mkb::FspInstance> d_inst;
    mkb::DeviceArray<double> d_rates, d_out;
    mkb::DeviceArray<mkb::FspOutcome> d_outcome;
    mkb::DeviceArray<int> d_queue;
    mkb::DeviceArray<double> work;
    mkb::DeviceArray<int> iwork;
    int workspace_blocks = 0;               // blocks the workspace holds
    int threads = 512;
    int blocks = 0;                         // 0: every block that fits
    int sms = 0;
};

namespace {

using mkb::Error;

int status_code(int device_status) {
    switch (device_status) {
    case 0:
        return MK_OK;
    case 1:
        return MK_ETOLERANCE;
    case 2:
        return MK_ENOTCONV;
    default:
        return MK_ENAN;
    }
}

const char *status_text(int device_status) {
    switch (device_status) {
    case 1:
        return "expv: the requested tolerance is too high";
    case 2:
        return "stopped before final_time (max_steps or the substep limit)";
    default:
        return "non-finite Krylov vector";
    }
}

std::int64_t box_size(int S, const int *bounds) {
    std::int64_t size = 1;
    for (int s = 0; s < S; ++s) {
        if (bounds[s] < 0) {
            throw Error(MK_EINVAL, "fsp: negative box bound");
        }
        size *= static_cast<std::int64_t>(bounds[s]) + 1;
        if (size > (std::int64_t(1) << 30)) {
            throw Error(MK_EOVERFLOW, "fsp: box too large (more than 2^30 states)");
        }
    }
    return size;
}

void check_options(const mk_fsp_options &o) {
    MK_REQUIRE(o.krylov_dim >= 1 && o.krylov_dim <= mkb::kFspMaxKrylov,
               "fsp: krylov_dim must be in 1..30");
    MK_REQUIRE(o.layers >= 0, "fsp: layers must be >= 0");
    MK_REQUIRE(o.max_steps >= 0, "fsp: max_steps must be >= 0");
    MK_REQUIRE(std::isfinite(o.tolerance) && std::isfinite(o.initial_step) &&
                   std::isfinite(o.step_growth) && std::isfinite(o.krylov_tol) &&
                   o.krylov_tol > 0.0,
               "fsp: options must be finite, krylov_tol > 0");
    MK_REQUIRE(o.method == 0 || o.method == 1, "fsp: method must be 0 (Krylov) or 1 (adaptive)");
    MK_REQUIRE(std::isfinite(o.step_scale) && o.step_scale > 0.0 && std::isfinite(o.prune_fraction) &&
                   o.prune_fraction >= 0.0 && std::isfinite(o.flux_tolerance) &&
                   std::isfinite(o.min_probability),
               "fsp: adaptive options must be finite, step_scale > 0, prune_fraction >= 0");
}

int sm_count() {
    int dev = 0, sms = 0;
    mkb::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    mkb::check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                    "cudaDeviceGetAttribute");
    return sms;
}

// blocks a launch of this shape uses
int resolve_blocks(const mk_fsp_batch_s &b, int threads, int blocks) {
    if (blocks <= 0) {
        const int per_sm = mkb::fsp_blocks_per_sm(threads);
        if (per_sm <= 0) {
            throw Error(MK_ECUDA, "fsp: the kernel does not fit on an SM");
        }
        blocks = per_sm * b.sms;
    }
    return std::max(1, std::min(blocks, b.n));
}

void ensure_workspace(mk_fsp_batch_s &b, int blocks) {
    if (blocks <= b.workspace_blocks) {
        return;
    }
    b.work.resize(static_cast<std::size_t>(blocks) * mkb::fsp_work_doubles(b.cap, b.rmax));
    b.iwork.resize(static_cast<std::size_t>(blocks) * mkb::fsp_work_ints(b.cap, b.rmax));
    b.workspace_blocks = blocks;
}

// blocks is the launch's total; the shared arena is what that many blocks per SM leave
void launch(mk_fsp_batch_s &b, const mkb::FspInstance *d_inst, int n, int threads, int blocks,
            cudaStream_t stream) {
    const int per_sm = std::max(1, (blocks + b.sms - 1) / b.sms);
    const std::size_t arena = mkb::fsp_arena_bytes(threads, per_sm);
    blocks = std::max(1, std::min(blocks, n));
    ensure_workspace(b, blocks);
    mkb::check_cuda(cudaMemsetAsync(b.d_queue.get(), 0, sizeof(int), stream), "fsp queue reset");
    mkb::FspBatchView v;
    v.inst = d_inst;
    v.n = n;
    v.rates = b.d_rates.get();
    v.out = b.d_out.get();
    v.outcome = b.d_outcome.get();
    v.queue = b.d_queue.get();
    v.work = b.work.get();
    v.iwork = b.iwork.get();
    v.cap = b.cap;
    v.rmax = b.rmax;
    v.arena_bytes = arena;
    mkb::check_cuda(mkb::launch_fsp_batch(v, threads, blocks, stream), "fsp kernel launch");
}

} // namespace

extern "C" {

void mk_fsp_options_default(mk_fsp_options *opt) {
    if (!opt) {
        return;
    }
    opt->tolerance = 1e-6;
    opt->initial_step = 1.0;
    opt->step_growth = 2.0;
    opt->drop_probability = 1e-10;
    opt->drop_derivative = 1e-16;
    opt->layers = 1;
    opt->krylov_dim = 30;
    opt->max_steps = std::int64_t(1) << 28;
    opt->krylov_tol = 1e-8;
    opt->method = 0;
    opt->step_scale = 1.0;
    opt->prune_fraction = 0.1;
    opt->flux_tolerance = 1e-6;
    opt->min_probability = 0.0;
}

int mk_fsp_box_size(int n_species, const int *bounds, int64_t *size) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(bounds && size, "null argument");
        MK_REQUIRE(n_species >= 1 && n_species <= mkb::kFspMaxSpecies, "fsp: 1..4 species");
        *size = box_size(n_species, bounds);
    });
}

int mk_fsp_batch_create(int n, const mk_fsp_problem *problems, mk_fsp_batch *out) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(out && (n == 0 || problems), "null argument");
        MK_REQUIRE(n >= 1, "fsp: empty batch");
        auto b = std::make_unique<mk_fsp_batch_s>();
        b->n = n;
        std::vector<mkb::FspInstance> inst(n);
        std::vector<std::int64_t> rate_offset(n);
        b->out_offset.resize(n);
        std::int64_t rate_total = 0;
        for (int k = 0; k < n; ++k) {
            const mk_fsp_problem &p = problems[k];
            const std::string where = "fsp instance " + std::to_string(k) + ": ";
            MK_REQUIRE(p.n_species >= 1 && p.n_species <= mkb::kFspMaxSpecies,
                       where + "1..4 species");
            MK_REQUIRE(p.n_reactions >= 0 && p.n_reactions <= mkb::kFspMaxReactions,
                       where + "0..16 reactions");
            MK_REQUIRE(p.bounds && p.initial && (p.n_reactions == 0 || (p.change && p.rates)),
                       where + "null array");
            MK_REQUIRE(std::isfinite(p.final_time) && p.final_time >= 0.0,
                       where + "final_time must be finite and >= 0");
            check_options(p.options);
            mkb::FspInstance &I = inst[k];
            I.S = p.n_species;
            I.R = p.n_reactions;
            const std::int64_t box = box_size(p.n_species, p.bounds);
            if (box * std::max(p.n_reactions, 1) >= (std::int64_t(1) << 31)) {
                throw Error(MK_EOVERFLOW,
                            where + "box size x reactions must stay below 2^31");
            }
            I.box = static_cast<int>(box);
            std::int64_t stride = 1;
            for (int s = p.n_species - 1; s >= 0; --s) {
                I.bound[s] = p.bounds[s];
                I.stride[s] = static_cast<int>(stride);
                stride *= p.bounds[s] + 1;
            }
            std::int64_t initial = 0;
            for (int s = 0; s < p.n_species; ++s) {
                MK_REQUIRE(p.initial[s] >= 0 && p.initial[s] <= p.bounds[s],
                           where + "the initial state must lie in the box");
                initial += static_cast<std::int64_t>(p.initial[s]) * I.stride[s];
            }
            I.initial = static_cast<int>(initial);
            for (int r = 0; r < p.n_reactions; ++r) {
                for (int s = 0; s < p.n_species; ++s) {
                    I.change[r][s] = p.change[r * p.n_species + s];
                }
            }
            I.layers = p.options.layers;
            I.krylov_dim = p.options.krylov_dim;
            I.index = k;
            I.max_steps = p.options.max_steps;
            I.final_time = p.final_time;
            I.tolerance = p.options.tolerance;
            I.initial_step = p.options.initial_step;
            I.step_growth = p.options.step_growth;
            I.drop_probability = p.options.drop_probability;
            I.drop_derivative = p.options.drop_derivative;
            I.krylov_tol = p.options.krylov_tol;
            I.method = p.options.method;
            I.step_scale = p.options.step_scale;
            I.prune_fraction = p.options.prune_fraction;
            I.flux_tolerance = p.options.flux_tolerance;
            I.min_probability = p.options.min_probability;
            rate_offset[k] = rate_total;
            I.rate_offset = rate_total;
            rate_total += box * p.n_reactions;
            b->out_offset[k] = b->total_box;
            I.out_offset = b->total_box;
            b->total_box += box;
            b->cap = std::max(b->cap, box);
            b->rmax = std::max(b->rmax, p.n_reactions);
        }
        // the kernel packs vectors at the support size rounded up to 4 states
        b->cap = (b->cap + 3) & ~std::int64_t(3);
        std::vector<double> rates(static_cast<std::size_t>(std::max<std::int64_t>(rate_total, 1)),
                                  0.0);
        for (int k = 0; k < n; ++k) {
            const std::int64_t len = static_cast<std::int64_t>(inst[k].box) * inst[k].R;
            if (len > 0) {
                std::copy(problems[k].rates, problems[k].rates + len, rates.begin() + rate_offset[k]);
            }
        }
        // largest box first, so the long instances start early and short ones fill the tail
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int c) { return inst[a].box > inst[c].box; });
        b->inst.reserve(n);
        for (int k : order) {
            b->inst.push_back(inst[k]);
        }
        b->d_inst.upload(b->inst);
        b->d_rates.upload(rates);
        b->d_out.resize(static_cast<std::size_t>(b->total_box));
        b->d_outcome.resize(static_cast<std::size_t>(n));
        b->d_queue.resize(1);
        b->sms = sm_count();
        *out = b.release();
    });
}

void mk_fsp_batch_destroy(mk_fsp_batch batch) { delete batch; }

int mk_fsp_batch_output_size(mk_fsp_batch batch, int64_t *total, int64_t *h_offsets) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(batch && total, "null argument");
        *total = batch->total_box;
        if (h_offsets) {
            std::copy(batch->out_offset.begin(), batch->out_offset.end(), h_offsets);
        }
    });
}

int mk_fsp_batch_set_shape(mk_fsp_batch batch, int threads, int blocks) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(batch, "null argument");
        MK_REQUIRE(threads == 128 || threads == 256 || threads == 512,
                   "fsp: threads must be 128, 256 or 512");
        MK_REQUIRE(blocks >= 0, "fsp: blocks must be >= 0");
        batch->threads = threads;
        batch->blocks = blocks;
    });
}

int mk_fsp_batch_get_shape(mk_fsp_batch batch, int *threads, int *blocks) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(batch && threads && blocks, "null argument");
        *threads = batch->threads;
        *blocks = resolve_blocks(*batch, batch->threads, batch->blocks);
    });
}

int mk_fsp_batch_autotune(mk_fsp_batch batch, int sample, void *stream) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(batch, "null argument");
        MK_REQUIRE(sample >= 0, "fsp: sample must be >= 0");
        const cudaStream_t st = mkb::capi::as_stream(stream);
        // evenly spaced instances of the queue, so the sample keeps the size mix
        const int n = batch->n;
        const int m = sample == 0 ? n : std::min(sample, n);
        std::vector<mkb::FspInstance> sub;
        sub.reserve(m);
        for (int q = 0; q < m; ++q) {
            sub.push_back(batch->inst[static_cast<std::size_t>(q) * n / m]);
        }
        mkb::DeviceArray<mkb::FspInstance> d_sub;
        d_sub.upload(sub);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        mkb::check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        mkb::check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        float best = -1.0f;
        int best_threads = batch->threads, best_blocks = batch->blocks;
        try {
            for (int threads : mkb::kFspShapes) {
                const int per_sm = mkb::fsp_blocks_per_sm(threads);
                for (int k = 1; k <= per_sm; ++k) {
                    const int blocks = std::min(k * batch->sms, m);
                    launch(*batch, d_sub.get(), m, threads, blocks, st);  // warm-up
                    mkb::check_cuda(cudaEventRecord(e0, st), "cudaEventRecord");
                    launch(*batch, d_sub.get(), m, threads, blocks, st);
                    mkb::check_cuda(cudaEventRecord(e1, st), "cudaEventRecord");
                    mkb::check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
                    float ms = 0.0f;
                    mkb::check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                    if (best < 0.0f || ms < best) {
                        best = ms;
                        best_threads = threads;
                        best_blocks = k * batch->sms;
                    }
                    if (blocks >= m) {
                        break;
                    }
                }
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        batch->threads = best_threads;
        batch->blocks = best_blocks;
    });
}

int mk_fsp_batch_run(mk_fsp_batch batch, void *stream) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(batch, "null argument");
        const int blocks = resolve_blocks(*batch, batch->threads, batch->blocks);
        launch(*batch, batch->d_inst.get(), batch->n, batch->threads, blocks,
               mkb::capi::as_stream(stream));
    });
}

int mk_fsp_batch_device_output(mk_fsp_batch batch, const double **d_out) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(batch && d_out, "null argument");
        *d_out = batch->d_out.get();
    });
}

int mk_fsp_batch_results(mk_fsp_batch batch, double *h_out, mk_fsp_result *results,
                         void *stream) {
    int first_failure = MK_OK;
    const int rc = mkb::capi::guarded([&] {
        MK_REQUIRE(batch && results, "null argument");
        const cudaStream_t st = mkb::capi::as_stream(stream);
        std::vector<mkb::FspOutcome> outcome(batch->n);
        mkb::check_cuda(cudaMemcpyAsync(outcome.data(), batch->d_outcome.get(),
                                        sizeof(mkb::FspOutcome) * batch->n,
                                        cudaMemcpyDeviceToHost, st),
                        "fsp results copy");
        if (h_out) {
            mkb::check_cuda(cudaMemcpyAsync(h_out, batch->d_out.get(),
                                            sizeof(double) * batch->total_box,
                                            cudaMemcpyDeviceToHost, st),
                            "fsp output copy");
        }
        mkb::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        for (int k = 0; k < batch->n; ++k) {
            mk_fsp_result &r = results[k];
            r.time = outcome[k].time;
            r.attempts = outcome[k].attempts;
            r.accepted = outcome[k].accepted;
            r.support = outcome[k].support;
            r.substeps = outcome[k].substeps;
            r.applies = outcome[k].applies;
            r.status = status_code(outcome[k].status);
            r.clipped = outcome[k].clipped;
            if (r.status != MK_OK && first_failure == MK_OK) {
                first_failure = r.status;
                mkb::capi::g_last_error =
                    "fsp instance " + std::to_string(k) + ": " + status_text(outcome[k].status);
            }
        }
    });
    return rc != MK_OK ? rc : first_failure;
}

int mk_fsp_krylov_batch(int n, const mk_fsp_problem *problems, double *h_out,
                        mk_fsp_result *results, void *stream) {
    mk_fsp_batch batch = nullptr;
    int rc = mk_fsp_batch_create(n, problems, &batch);
    if (rc != MK_OK) {
        return rc;
    }
    rc = mk_fsp_batch_run(batch, stream);
    if (rc == MK_OK) {
        rc = mk_fsp_batch_results(batch, h_out, results, stream);
    }
    mk_fsp_batch_destroy(batch);
    return rc;
}

} // extern "C"
