// The resolvent request loop behind mk_server_* (include/markovkit_b200.h, "Serving").
//
// Requests (sI - Q) x = b on registered problems (a population space and an RDME model) are
// queued first come, first served. Each of `slots` worker threads owns one CUDA stream and takes
// the next request when it is free, so up to `slots` solves run on the device at once and their
// kernels overlap. A solve runs on a resident solver for (problem, shift): generator, sector
// multigrid (FP32 inside flexible GMRES, or FP64 inside plain GMRES), Krylov workspace and device
// b and x, kept after the solve for the next request with the same key. Admission is by HBM
// footprint: before a new resident solver is built, idle ones are evicted least recently used
// first until the estimate fits the budget; if the remaining ones are all busy, the worker waits
// until one finishes. A request whose footprint alone exceeds the budget fails with MK_ENOMEM.
// Latency is measured from submit to the device->host copy of x having completed.
#include "capi_internal.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

// smoother -1: red-black Gauss-Seidel where its colour passes pay for themselves (one species
// of at most two molecules per state: 20 against 26 iterations at about the cost of a Jacobi
// cycle on a 4096-voxel box), weighted Jacobi elsewhere (with longer molecule lists or more
// species a colour pass costs as much as a whole Jacobi sweep, and the iterations saved do not
// cover it)
int auto_smoother(const mkb::Space &sp) {
    const int cap = *std::max_element(sp.limits.begin(), sp.limits.end());
    return sp.S == 1 && cap <= 2 ? 1 : 0;
}

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Problem {
    std::unique_ptr<mkb::Space> space;
    std::unique_ptr<mkb::Model> model;
    std::int64_t n = 0;
};

struct Resident {
    int problem = -1;
    double shift = 0.0;
    int width = 1;                          // requests one solve serves
    std::unique_ptr<mkb::Generator> gen;
    std::unique_ptr<mkb::Multigrid> mg;
    std::unique_ptr<mkb::Krylov> ws;        // batch width 1
    std::unique_ptr<mkb::KrylovBatch> wsb;  // batch width > 1
    std::int64_t ld = 0;                    // stride of the columns of b and x
    mkb::DeviceArray<double> b, x;
    std::size_t bytes = 0;   // admitted footprint
    bool busy = false;
    bool built = false;
    std::uint64_t last_used = 0;
};

struct Request {
    std::int64_t ticket = 0;
    int problem = -1;
    double shift = 0.0;
    const double *h_b = nullptr;
    double *h_x = nullptr;
    Clock::time_point submitted;
};

} // namespace

struct mk_server_s {
    mk_server_options opt{};
    int device = 0;
    std::size_t budget = 0;
    std::vector<std::unique_ptr<Problem>> problems;
    std::vector<std::unique_ptr<Resident>> resident;
    std::size_t resident_bytes = 0;
    std::deque<Request> queue;
    std::unordered_map<std::int64_t, mk_server_result> done;
    std::vector<double> latencies;
    std::int64_t next_ticket = 1;
    std::int64_t in_flight = 0;
    std::int64_t evictions = 0;
    std::int64_t memory_waits = 0;
    std::uint64_t tick = 0;
    Clock::time_point first_submit{}, last_done{};
    bool any_submit = false;
    bool stopping = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_mem, cv_done;
    std::vector<std::thread> workers;

    // bytes charged for a resident solver of n states that solves `width` requests together
    [[nodiscard]] std::size_t footprint(std::int64_t n, int width) const {
        const std::int64_t m = opt.restart;
        const bool flexible = opt.precision == 1 || width > 1;
        const std::int64_t krylov = (m + 1) + (flexible ? m : 0) + 7; // + w, r, t, b, x
        const std::int64_t mg = opt.precision == 1 ? 48 : 96;        // level vectors
        const std::int64_t terminal = std::min<std::int64_t>(opt.coarsest_size, 8192);
        return static_cast<std::size_t>(n) * static_cast<std::size_t>((8 * krylov + mg) * width) +
               static_cast<std::size_t>(terminal * terminal * 12) + (std::size_t(16) << 20);
    }

    // the batch width of a problem's resident solvers: the widest up to opt.batch whose
    // footprint leaves every slot an equal share of the budget, else 1 (large spaces, such as a
    // 186M-state box, are served one request at a time instead of being refused)
    [[nodiscard]] int width_for(std::int64_t n) const {
        for (int w = opt.batch; w > 1; --w) {
            if (footprint(n, w) <= budget / static_cast<std::size_t>(opt.slots)) {
                return w;
            }
        }
        return 1;
    }

    [[nodiscard]] std::size_t footprint(std::int64_t n) const {
        return footprint(n, width_for(n));
    }

    void finish(const Request &rq, mk_server_result r, Clock::time_point started) {
        const auto now = Clock::now();
        r.ticket = rq.ticket;
        r.latency_ms = ms_between(rq.submitted, now);
        r.queue_ms = ms_between(rq.submitted, started);
        r.solve_ms = ms_between(started, now);
        std::lock_guard<std::mutex> lock(mu);
        done[rq.ticket] = r;
        if (r.status == MK_OK || r.status == MK_ENOTCONV) {
            latencies.push_back(r.latency_ms);
        }
        last_done = now;
        --in_flight;
        cv_done.notify_all();
    }

    // pick or reserve the resident solver for a request; nullptr: rejected (result recorded)
    Resident *admit(const Request &rq, std::unique_lock<std::mutex> &lock) {
        for (auto &r : resident) {
            if (!r->busy && r->built && r->problem == rq.problem && r->shift == rq.shift) {
                r->busy = true;
                return r.get();
            }
        }
        const std::size_t need = footprint(problems[rq.problem]->n);
        if (need > budget) {
            return nullptr;
        }
        bool waited = false;
        while (resident_bytes + need > budget) {
            auto victim = resident.end();
            for (auto it = resident.begin(); it != resident.end(); ++it) {
                if (!(*it)->busy && (victim == resident.end() || (*it)->last_used < (*victim)->last_used)) {
                    victim = it;
                }
            }
            if (victim != resident.end()) {
                resident_bytes -= (*victim)->bytes;
                resident.erase(victim);
                ++evictions;
                continue;
            }
            if (!waited) {
                ++memory_waits;
                waited = true;
            }
            cv_mem.wait(lock);
            if (stopping) {
                return nullptr;
            }
            // a solver for this key may have been freed meanwhile
            for (auto &r : resident) {
                if (!r->busy && r->built && r->problem == rq.problem && r->shift == rq.shift) {
                    r->busy = true;
                    return r.get();
                }
            }
        }
        auto r = std::make_unique<Resident>();
        r->problem = rq.problem;
        r->shift = rq.shift;
        r->width = width_for(problems[rq.problem]->n);
        r->bytes = need;
        r->busy = true;
        resident_bytes += need;
        resident.push_back(std::move(r));
        return resident.back().get();
    }

    void release(Resident *r, bool keep) {
        std::lock_guard<std::mutex> lock(mu);
        r->busy = false;
        r->last_used = ++tick;
        if (!keep) {
            for (auto it = resident.begin(); it != resident.end(); ++it) {
                if (it->get() == r) {
                    resident_bytes -= r->bytes;
                    resident.erase(it);
                    break;
                }
            }
        }
        cv_mem.notify_all();
    }

    void worker() {
        cudaSetDevice(device);
        cudaStream_t stream = nullptr;
        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        while (true) {
            // the oldest request, and queued requests for the same (problem, shift) up to the
            // batch width: they share one resident solver and one batched solve
            std::vector<Request> batch;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait(lock, [&] { return stopping || !queue.empty(); });
                if (stopping && queue.empty()) {
                    break;
                }
                batch.push_back(queue.front());
                queue.pop_front();
                const int width = width_for(problems[batch[0].problem]->n);
                for (auto it = queue.begin(); it != queue.end() &&
                                              static_cast<int>(batch.size()) < width;) {
                    if (it->problem == batch[0].problem && it->shift == batch[0].shift) {
                        batch.push_back(*it);
                        it = queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            const Request &rq = batch[0];
            const int nb = static_cast<int>(batch.size());
            std::vector<mk_server_result> res(nb);
            Resident *r = nullptr;
            {
                std::unique_lock<std::mutex> lock(mu);
                r = admit(rq, lock);
            }
            const auto started = Clock::now(); // a slot and the memory are ours from here
            if (!r) {
                for (int c = 0; c < nb; ++c) {
                    res[c].status = MK_ENOMEM;
                    finish(batch[c], res[c], started);
                }
                continue;
            }
            bool keep = true;
            try {
                const Problem &p = *problems[rq.problem];
                if (!r->built) {
                    r->gen = std::make_unique<mkb::Generator>(*p.space, *p.model, true);
                    mkb::MultigridOptions mo;
                    mo.precision = opt.precision == 1 ? 1 : 0;
                    mo.smoother = opt.smoother >= 0 ? opt.smoother : auto_smoother(*p.space);
                    mo.coarsest_size = opt.coarsest_size;
                    mo.batch = r->width;
                    r->mg = std::make_unique<mkb::Multigrid>(*p.space, *p.model, rq.shift, mo);
                    if (r->width == 1) {
                        r->ws = std::make_unique<mkb::Krylov>(p.n, opt.restart, opt.precision == 1);
                        r->ld = p.n;
                    } else {
                        r->wsb = std::make_unique<mkb::KrylovBatch>(p.n, opt.restart, r->width);
                        r->ld = r->wsb->ld;
                    }
                    r->b.resize(static_cast<std::size_t>(r->ld) * r->width);
                    r->x.resize(static_cast<std::size_t>(r->ld) * r->width);
                    r->built = true;
                }
                std::vector<double> tol(nb), bnorm(nb);
                for (int c = 0; c < nb; ++c) {
                    double s = 0.0;
                    for (std::int64_t i = 0; i < p.n; ++i) {
                        s += batch[c].h_b[i] * batch[c].h_b[i];
                    }
                    bnorm[c] = std::sqrt(s);
                    tol[c] = opt.rel_tolerance * bnorm[c];
                    mkb::check_cuda(cudaMemcpyAsync(r->b.get() + c * r->ld, batch[c].h_b,
                                                    sizeof(double) * p.n, cudaMemcpyHostToDevice,
                                                    stream),
                                    "request b copy");
                }
                mkb::check_cuda(cudaMemsetAsync(r->x.get(), 0, sizeof(double) * r->ld * nb, stream),
                                "request x reset");
                mkb::GmresOptions go;
                go.max_iterations = opt.max_iterations;
                go.restart = opt.restart;
                go.flexible = opt.precision == 1 ? 1 : 0;
                std::vector<mkb::SolverResult> sr;
                if (r->ws) {
                    go.tolerance = tol[0];
                    sr.push_back(mkb::gmres(*r->gen, rq.shift, r->mg.get(), r->b.get(), r->x.get(),
                                            go, *r->ws, stream));
                } else {
                    sr = mkb::gmres_batch(*r->gen, rq.shift, *r->mg, r->b.get(), r->x.get(), nb,
                                          tol.data(), go, *r->wsb, stream);
                }
                for (int c = 0; c < nb; ++c) {
                    mkb::check_cuda(cudaMemcpyAsync(batch[c].h_x, r->x.get() + c * r->ld,
                                                    sizeof(double) * p.n, cudaMemcpyDeviceToHost,
                                                    stream),
                                    "request x copy");
                }
                mkb::check_cuda(cudaStreamSynchronize(stream), "request sync");
                for (int c = 0; c < nb; ++c) {
                    res[c].iterations = sr[c].iterations;
                    res[c].residual = sr[c].residual / (bnorm[c] > 0.0 ? bnorm[c] : 1.0);
                    res[c].status = sr[c].converged ? MK_OK
                                                    : (sr[c].status != 0 ? sr[c].status : MK_ENOTCONV);
                    res[c].batched = nb;
                }
            } catch (const mkb::Error &e) {
                for (auto &x : res) {
                    x.status = e.code;
                }
                keep = false;
            } catch (const std::bad_alloc &) {
                for (auto &x : res) {
                    x.status = MK_ENOMEM;
                }
                keep = false;
            } catch (const std::exception &) {
                for (auto &x : res) {
                    x.status = MK_ECUDA;
                }
                keep = false;
            }
            release(r, keep && r->built);
            for (int c = 0; c < nb; ++c) {
                finish(batch[c], res[c], started);
            }
        }
        cudaStreamDestroy(stream);
    }
};

extern "C" {

void mk_server_options_default(mk_server_options *opt) {
    if (!opt) {
        return;
    }
    opt->slots = 4;
    opt->hbm_budget = 0;
    opt->precision = 1;
    opt->smoother = 0;
    opt->restart = 30;
    opt->max_iterations = 5000;
    opt->rel_tolerance = 1e-10;
    opt->batch = 4;
    opt->coarsest_size = 256;
}

int mk_server_create(const mk_server_options *opt, mk_server *out) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(opt && out, "null argument");
        MK_REQUIRE(opt->slots >= 1 && opt->slots <= 64, "server: slots must be in 1..64");
        MK_REQUIRE(opt->restart >= 1 && opt->restart <= 64, "server: restart must be in 1..64");
        MK_REQUIRE(opt->precision == 0 || opt->precision == 1, "server: precision is 0 or 1");
        MK_REQUIRE(opt->smoother >= -1 && opt->smoother <= 2, "server: smoother is -1, 0, 1 or 2");
        MK_REQUIRE(opt->max_iterations >= 1 && opt->rel_tolerance > 0.0,
                   "server: max_iterations >= 1 and rel_tolerance > 0");
        MK_REQUIRE(opt->batch >= 1 && opt->batch <= mkb::kRowBatch, "server: batch must be in 1..4");
        MK_REQUIRE(opt->coarsest_size >= 1 && opt->coarsest_size <= 8192,
                   "server: coarsest_size must be in 1..8192");
        auto s = std::make_unique<mk_server_s>();
        s->opt = *opt;
        mkb::check_cuda(cudaGetDevice(&s->device), "cudaGetDevice");
        std::size_t free_b = 0, total_b = 0;
        mkb::check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        s->budget = opt->hbm_budget ? opt->hbm_budget : free_b / 10 * 8;
        for (int k = 0; k < opt->slots; ++k) {
            s->workers.emplace_back([srv = s.get()] { srv->worker(); });
        }
        *out = s.release();
    });
}

void mk_server_destroy(mk_server server) {
    if (!server) {
        return;
    }
    {
        std::lock_guard<std::mutex> lock(server->mu);
        server->stopping = true;
    }
    server->cv_work.notify_all();
    server->cv_mem.notify_all();
    for (auto &t : server->workers) {
        t.join();
    }
    delete server;
}

int mk_server_register(mk_server server, mk_space space, mk_model model, int *problem) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(server && space && model && problem, "null argument");
        MK_REQUIRE(space->space->V == model->model->V,
                   "server: the space and the model have different voxel counts");
        auto p = std::make_unique<Problem>();
        const mkb::Space &sp = *space->space;
        p->space = mkb::Space::make(sp.V, sp.limits, sp.is_box);
        p->model = std::make_unique<mkb::Model>(*model->model);
        p->model->validate();
        p->n = p->space->n;
        std::lock_guard<std::mutex> lock(server->mu);
        server->problems.push_back(std::move(p));
        *problem = static_cast<int>(server->problems.size()) - 1;
    });
}

int mk_server_submit(mk_server server, int problem, double shift, const double *h_b, double *h_x,
                     int64_t *ticket) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(server && h_b && h_x && ticket, "null argument");
        MK_REQUIRE(std::isfinite(shift) && shift > 0.0, "server: shift must be finite and > 0");
        std::lock_guard<std::mutex> lock(server->mu);
        MK_REQUIRE(problem >= 0 && problem < static_cast<int>(server->problems.size()),
                   "server: unknown problem");
        MK_REQUIRE(!server->stopping, "server: stopping");
        Request rq;
        rq.ticket = server->next_ticket++;
        rq.problem = problem;
        rq.shift = shift;
        rq.h_b = h_b;
        rq.h_x = h_x;
        rq.submitted = Clock::now();
        if (!server->any_submit) {
            server->first_submit = rq.submitted;
            server->any_submit = true;
        }
        server->queue.push_back(rq);
        ++server->in_flight;
        *ticket = rq.ticket;
        server->cv_work.notify_one();
    });
}

int mk_server_wait(mk_server server, int64_t ticket, mk_server_result *result) {
    int status = MK_OK;
    const int rc = mkb::capi::guarded([&] {
        MK_REQUIRE(server && result, "null argument");
        std::unique_lock<std::mutex> lock(server->mu);
        MK_REQUIRE(ticket >= 1 && ticket < server->next_ticket, "server: unknown ticket");
        server->cv_done.wait(lock, [&] { return server->done.count(ticket) > 0; });
        *result = server->done[ticket];
        status = result->status;
    });
    if (rc != MK_OK) {
        return rc;
    }
    if (status != MK_OK) {
        mkb::capi::g_last_error = "server: request " + std::to_string(ticket) + " ended with status " +
                                  std::to_string(status);
    }
    return status;
}

int mk_server_wait_for(mk_server server, int64_t ticket, double timeout_ms,
                       mk_server_result *result) {
    int status = MK_OK;
    const int rc = mkb::capi::guarded([&] {
        MK_REQUIRE(server && result, "null argument");
        MK_REQUIRE(timeout_ms >= 0.0 && std::isfinite(timeout_ms), "server: timeout must be finite and >= 0");
        std::unique_lock<std::mutex> lock(server->mu);
        MK_REQUIRE(ticket >= 1 && ticket < server->next_ticket, "server: unknown ticket");
        const auto limit = std::chrono::duration<double, std::milli>(timeout_ms);
        if (!server->cv_done.wait_for(lock, limit, [&] { return server->done.count(ticket) > 0; })) {
            throw mkb::Error(MK_ETIMEOUT, "server: request " + std::to_string(ticket) +
                                              " not done within the timeout");
        }
        *result = server->done[ticket];
        status = result->status;
    });
    if (rc != MK_OK) {
        return rc;
    }
    if (status != MK_OK) {
        mkb::capi::g_last_error = "server: request " + std::to_string(ticket) + " ended with status " +
                                  std::to_string(status);
    }
    return status;
}

int mk_server_cancel(mk_server server, int64_t ticket) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(server, "null argument");
        std::lock_guard<std::mutex> lock(server->mu);
        MK_REQUIRE(ticket >= 1 && ticket < server->next_ticket, "server: unknown ticket");
        auto it = std::find_if(server->queue.begin(), server->queue.end(),
                               [&](const Request &rq) { return rq.ticket == ticket; });
        MK_REQUIRE(it != server->queue.end(), "server: the request has already started or finished");
        mk_server_result r{};
        r.ticket = ticket;
        r.status = MK_ECANCELED;
        r.latency_ms = r.queue_ms = ms_between(it->submitted, Clock::now());
        server->queue.erase(it);
        server->done[ticket] = r;
        --server->in_flight;
        server->cv_done.notify_all();
    });
}

int mk_server_drain(mk_server server) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(server, "null argument");
        std::unique_lock<std::mutex> lock(server->mu);
        server->cv_done.wait(lock, [&] { return server->in_flight == 0; });
    });
}

int mk_server_stats_get(mk_server server, mk_server_stats *stats) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(server && stats, "null argument");
        std::lock_guard<std::mutex> lock(server->mu);
        std::vector<double> lat = server->latencies;
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double q) {
            if (lat.empty()) {
                return 0.0;
            }
            const std::size_t k = static_cast<std::size_t>(
                std::llround(q * static_cast<double>(lat.size() - 1)));
            return lat[std::min(k, lat.size() - 1)];
        };
        stats->completed = static_cast<std::int64_t>(lat.size());
        stats->p50_ms = pct(0.50);
        stats->p99_ms = pct(0.99);
        const double span = server->any_submit ? ms_between(server->first_submit, server->last_done) : 0.0;
        stats->solves_per_s = span > 0.0 ? 1e3 * static_cast<double>(lat.size()) / span : 0.0;
        stats->resident_bytes = server->resident_bytes;
        stats->budget_bytes = server->budget;
        stats->resident_solvers = static_cast<std::int64_t>(server->resident.size());
        stats->evictions = server->evictions;
        stats->memory_waits = server->memory_waits;
    });
}

int mk_server_footprint(mk_server server, int problem, size_t *bytes) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(server && bytes, "null argument");
        std::lock_guard<std::mutex> lock(server->mu);
        MK_REQUIRE(problem >= 0 && problem < static_cast<int>(server->problems.size()),
                   "server: unknown problem");
        *bytes = server->footprint(server->problems[problem]->n);
    });
}

} // extern "C"
