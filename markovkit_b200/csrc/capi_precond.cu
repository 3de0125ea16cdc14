// C ABI: the preconditioner handles of mk_solver_create_pc (precond.cuh) and generator::jumps.
#include "capi_internal.hpp"
#include "precond.cuh"

#include <vector>

using namespace mkb;
using mkb::capi::as_stream;
using mkb::capi::guarded;

int mk_precond_create_diagonal(int64_t n, const double *h_inverse_diagonal, mk_precond *out) {
    return guarded([&] {
        MK_REQUIRE(h_inverse_diagonal && out, "null argument");
        MK_REQUIRE(n >= 1, "empty preconditioner");
        auto h = std::make_unique<mk_precond_s>();
        h->pc = std::make_unique<DiagonalPreconditioner>(h_inverse_diagonal, n);
        *out = h.release();
    });
}

int mk_precond_create_ilu0(int64_t n, const int64_t *h_row_ptr, const int64_t *h_col,
                           const double *h_val, void *stream, mk_precond *out) {
    return guarded([&] {
        MK_REQUIRE(h_row_ptr && h_col && h_val && out, "null argument");
        auto h = std::make_unique<mk_precond_s>();
        h->pc = std::make_unique<Ilu0Preconditioner>(n, h_row_ptr, h_col, h_val, as_stream(stream));
        *out = h.release();
    });
}

int mk_precond_create_multigrid(mk_space space, mk_model model, double shift,
                                const mk_multigrid_options *opt, mk_precond *out) {
    return guarded([&] {
        MK_REQUIRE(space && model && out, "null argument");
        mk_multigrid mg = nullptr;
        const int rc = mk_multigrid_create(space, model, shift, opt, &mg);
        if (rc != MK_OK) {
            throw Error(rc, mk_last_error());
        }
        auto h = std::make_unique<mk_precond_s>();
        h->pc = std::move(mg->mg);
        mk_multigrid_destroy(mg);
        *out = h.release();
    });
}

int mk_precond_create_host(int64_t n, mk_precond_host_fn fn, void *ctx, mk_precond *out) {
    return guarded([&] {
        MK_REQUIRE(fn && out, "null argument");
        auto h = std::make_unique<mk_precond_s>();
        h->pc = std::make_unique<HostPreconditioner>(n, fn, ctx);
        *out = h.release();
    });
}

void mk_precond_destroy(mk_precond pc) { delete pc; }

int mk_precond_size(mk_precond pc, int64_t *n) {
    return guarded([&] {
        MK_REQUIRE(pc && n, "null argument");
        *n = pc->pc->n;
    });
}

int mk_precond_apply(mk_precond pc, const double *d_v, double *d_z, void *stream) {
    return guarded([&] {
        MK_REQUIRE(pc && d_v && d_z, "null argument");
        pc->pc->apply(d_v, d_z, as_stream(stream));
    });
}

int mk_precond_ilu0_schedule(mk_precond pc, int64_t *lower_levels, int64_t *upper_levels,
                             int64_t *launches_per_apply) {
    return guarded([&] {
        MK_REQUIRE(pc, "null argument");
        const auto *ilu = dynamic_cast<const Ilu0Preconditioner *>(pc->pc.get());
        MK_REQUIRE(ilu, "not an ILU(0) preconditioner");
        if (lower_levels) {
            *lower_levels = ilu->lower.levels();
        }
        if (upper_levels) {
            *upper_levels = ilu->upper.levels();
        }
        if (launches_per_apply) {
            *launches_per_apply =
                static_cast<int64_t>(ilu->lower.segments.size() + ilu->upper.segments.size());
        }
    });
}

// The jumps out of state j that stay in the space, in the reference's order
// (markovkit/generator.hpp:27-43 over reaction_diffusion::transitions,
// markovkit/rdme/reaction_diffusion.hpp:82-118): diffusion by voxel, edge, species with rate
// n * (D_s * w_e / volume_v); then reactions by voxel and reaction with the tabulated rate,
// skipping rates that are not positive and changes that leave a count negative.
int mk_generator_jumps(mk_generator gen, int64_t j, int64_t *h_to, double *h_rate,
                       int64_t capacity, int64_t *count) {
    return guarded([&] {
        MK_REQUIRE(gen && count, "null argument");
        MK_REQUIRE(capacity <= 0 || (h_to && h_rate), "null output arrays");
        const Space &sp = *gen->space;
        const Model &m = *gen->model;
        MK_REQUIRE(j >= 0 && j < sp.n, "state index out of range");
        const int V = sp.V, S = sp.S;
        std::vector<int> x(static_cast<std::size_t>(V) * S), y;
        sp.unrank(j, x.data());
        int64_t k = 0;
        auto emit = [&](double rate) {
            const std::int64_t i = sp.rank(y.data());
            if (i < 0) {
                return;
            }
            if (k < capacity) {
                h_to[k] = i;
                h_rate[k] = rate;
            }
            ++k;
        };
        for (int v = 0; v < V; ++v) {
            for (int e = m.nbr_ptr[v]; e < m.nbr_ptr[v + 1]; ++e) {
                const int w = m.nbr_idx[e];
                for (int s = 0; s < S; ++s) {
                    const int n = x[static_cast<std::size_t>(v) * S + s];
                    if (n == 0) {
                        continue;
                    }
                    y = x;
                    --y[static_cast<std::size_t>(v) * S + s];
                    ++y[static_cast<std::size_t>(w) * S + s];
                    emit(n * (m.diff[s] * m.nbr_w[e] / m.volumes[v]));
                }
            }
        }
        if (m.R > 0) {
            const int nt = m.ntuple();
            for (int v = 0; v < V; ++v) {
                int tuple = 0;
                for (int s = 0; s < S; ++s) {
                    const int c = x[static_cast<std::size_t>(v) * S + s];
                    MK_REQUIRE(c <= m.tmax[s], "a count exceeds the model's rate tables");
                    tuple = tuple * (m.tmax[s] + 1) + c;
                }
                const int vc = m.nvc > 1 ? m.vclass[v] : 0;
                for (int r = 0; r < m.R; ++r) {
                    const double rate =
                        m.rates[(static_cast<std::size_t>(r) * m.nvc + vc) * nt + tuple];
                    if (!(rate > 0.0)) {
                        continue;
                    }
                    y = x;
                    bool valid = true;
                    for (int s = 0; s < S; ++s) {
                        int &c = y[static_cast<std::size_t>(v) * S + s];
                        c += m.change[static_cast<std::size_t>(r) * S + s];
                        valid = valid && c >= 0;
                    }
                    if (valid) {
                        emit(rate);
                    }
                }
            }
        }
        *count = k;
    });
}
