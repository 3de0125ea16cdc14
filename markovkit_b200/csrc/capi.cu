// The C ABI (include/markovkit_b200.h) over the engine: handle bookkeeping, argument checks
// and the mapping of C++ errors to MK_* status codes.
#include "capi_internal.hpp"

#include <cmath>
#include <cstring>
#include <string>

using namespace mkb;
using mkb::capi::as_stream;
using mkb::capi::fail;
using mkb::capi::g_last_error;
using mkb::capi::guarded;
using mkb::capi::preconditioner_of;

extern "C" {

const char *mk_last_error(void) { return g_last_error.c_str(); }

int mk_version(void) { return 1; }

int mk_kernel_launches(uint64_t *count) {
    return guarded([&] {
        MK_REQUIRE(count, "null argument");
        *count = g_kernel_launches.load(std::memory_order_relaxed);
    });
}

int mk_set_row_path(int path) {
    return guarded([&] {
        MK_REQUIRE(path >= 0 && path <= 2,
                   "row path must be 0 (stencil where possible), 1 (general) or 2 (stencil, no pair strips)");
        set_row_path(path);
    });
}

int mk_device_alloc(size_t bytes, void **d_ptr) {
    return guarded([&] {
        MK_REQUIRE(d_ptr, "null output pointer");
        check_cuda(cudaMalloc(d_ptr, bytes), "cudaMalloc");
    });
}

int mk_device_free(void *d_ptr) {
    return guarded([&] { check_cuda(cudaFree(d_ptr), "cudaFree"); });
}

int mk_memcpy_h2d(void *d_dst, const void *h_src, size_t bytes, void *stream) {
    return guarded([&] {
        check_cuda(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, as_stream(stream)),
                   "copy");
    });
}

int mk_memcpy_d2h(void *h_dst, const void *d_src, size_t bytes, void *stream) {
    return guarded([&] {
        check_cuda(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)),
                   "copy");
        check_cuda(cudaStreamSynchronize(as_stream(stream)), "sync");
    });
}

int mk_stream_synchronize(void *stream) {
    return guarded([&] { check_cuda(cudaStreamSynchronize(as_stream(stream)), "sync"); });
}

// ---- spaces

static int create_space(int64_t n_voxels, int n_species, const int *limits, bool box,
                        mk_space *out) {
    return guarded([&] {
        MK_REQUIRE(out && limits, "null argument");
        MK_REQUIRE(n_voxels >= 1 && n_voxels <= (int64_t(1) << 30) && n_species >= 1,
                   "population state space needs a voxel and a species");
        std::vector<int> l(limits, limits + n_species);
        auto h = std::make_unique<mk_space_s>();
        h->space = Space::make(static_cast<int>(n_voxels), l, box);
        *out = h.release();
    });
}

int mk_space_create_box(int64_t n_voxels, int n_species, const int *max_totals, mk_space *out) {
    return create_space(n_voxels, n_species, max_totals, true, out);
}

int mk_space_create_sector(int64_t n_voxels, int n_species, const int *totals, mk_space *out) {
    return create_space(n_voxels, n_species, totals, false, out);
}

void mk_space_destroy(mk_space space) { delete space; }

int mk_space_size(mk_space space, int64_t *n) {
    return guarded([&] {
        MK_REQUIRE(space && n, "null argument");
        *n = space->space->n;
    });
}

int mk_space_n_sectors(mk_space space, int64_t *n_sectors) {
    return guarded([&] {
        MK_REQUIRE(space && n_sectors, "null argument");
        *n_sectors = static_cast<int64_t>(space->space->sectors.size());
    });
}

int mk_space_sector_begin(mk_space space, int64_t k, int64_t *begin) {
    return guarded([&] {
        MK_REQUIRE(space && begin, "null argument");
        const auto &s = space->space->sectors;
        MK_REQUIRE(k >= 0 && k <= static_cast<int64_t>(s.size()), "sector out of range");
        *begin = k == static_cast<int64_t>(s.size()) ? space->space->n : s[k].begin;
    });
}

int mk_space_sector_totals(mk_space space, int64_t k, int *totals) {
    return guarded([&] {
        MK_REQUIRE(space && totals, "null argument");
        const auto &s = space->space->sectors;
        MK_REQUIRE(k >= 0 && k < static_cast<int64_t>(s.size()), "sector out of range");
        for (int i = 0; i < space->space->S; ++i) {
            totals[i] = s[k].total[i];
        }
    });
}

int mk_space_find_sector(mk_space space, const int *totals, int64_t *k) {
    return guarded([&] {
        MK_REQUIRE(space && totals && k, "null argument");
        *k = space->space->find_sector(totals);
    });
}

int mk_space_sector_of(mk_space space, int64_t i, int64_t *k) {
    return guarded([&] {
        MK_REQUIRE(space && k, "null argument");
        MK_REQUIRE(i >= 0 && i < space->space->n, "state index out of range");
        *k = space->space->sector_of(i);
    });
}

int mk_space_find_host(mk_space space, const int *h_state, int64_t *index) {
    return guarded([&] {
        MK_REQUIRE(space && h_state && index, "null argument");
        *index = space->space->rank(h_state);
    });
}

int mk_space_state_host(mk_space space, int64_t i, int *h_state) {
    return guarded([&] {
        MK_REQUIRE(space && h_state, "null argument");
        space->space->unrank(i, h_state);
    });
}

int mk_space_rank(mk_space space, const int *d_states, int64_t count, int64_t *d_index,
                  void *stream) {
    return guarded([&] {
        MK_REQUIRE(space && (count == 0 || (d_states && d_index)), "null argument");
        const Space &sp = *space->space;
        MK_REQUIRE(sp.max_total <= 64, "device ranking supports totals up to 64");
        check_cuda(launch_rank(sp.binom->device_view(), sp.d_sectors.get(),
                               static_cast<int>(sp.sectors.size()), sp.d_limits.get(),
                               sp.is_box ? 1 : 0, sp.S, sp.V, d_states, count, d_index,
                               as_stream(stream)),
                   "rank");
    });
}

int mk_space_unrank(mk_space space, const int64_t *d_index, int64_t count, int *d_states,
                    void *stream) {
    return guarded([&] {
        MK_REQUIRE(space && (count == 0 || (d_states && d_index)), "null argument");
        const Space &sp = *space->space;
        MK_REQUIRE(sp.max_total <= 64, "device unranking supports totals up to 64");
        check_cuda(launch_unrank(sp.binom->device_view(), sp.d_sectors.get(),
                                 static_cast<int>(sp.sectors.size()), sp.S, sp.V, d_index, count,
                                 d_states, as_stream(stream)),
                   "unrank");
    });
}

// ---- models

int mk_model_create_grid(int dim, const int64_t *dims, const double *spacing, int n_species,
                         const double *diffusivities, mk_model *out) {
    return guarded([&] {
        MK_REQUIRE(out && dims && spacing && diffusivities, "null argument");
        MK_REQUIRE(n_species >= 1 && n_species <= kMaxSpecies, "1..4 species");
        std::vector<double> d(diffusivities, diffusivities + n_species);
        auto h = std::make_unique<mk_model_s>();
        h->model = Model::grid(dim, dims, spacing, d);
        *out = h.release();
    });
}

int mk_model_create_graph(int64_t n_voxels, const int64_t *nbr_ptr, const int64_t *nbr_idx,
                          const double *nbr_weight, const double *volumes, int n_species,
                          const double *diffusivities, mk_model *out) {
    return guarded([&] {
        MK_REQUIRE(out && nbr_ptr && volumes && diffusivities, "null argument");
        MK_REQUIRE(n_voxels >= 1 && n_voxels <= (int64_t(1) << 30), "bad voxel count");
        MK_REQUIRE(n_species >= 1 && n_species <= kMaxSpecies, "1..4 species");
        auto m = std::make_unique<Model>();
        m->V = static_cast<int>(n_voxels);
        m->S = n_species;
        const int64_t E = nbr_ptr[n_voxels];
        MK_REQUIRE(E >= 0 && E < (int64_t(1) << 31) && (E == 0 || (nbr_idx && nbr_weight)),
                   "bad edge list");
        m->nbr_ptr.assign(nbr_ptr, nbr_ptr + n_voxels + 1);
        m->nbr_idx.assign(nbr_idx, nbr_idx + E);
        m->nbr_w.assign(nbr_weight, nbr_weight + E);
        m->volumes.assign(volumes, volumes + n_voxels);
        m->diff.assign(diffusivities, diffusivities + n_species);
        m->validate();
        auto h = std::make_unique<mk_model_s>();
        h->model = std::move(m);
        *out = h.release();
    });
}

int mk_model_set_reactions(mk_model model, int n_reactions, const int *change,
                           const int *tuple_max, int n_volume_classes, const int *voxel_class,
                           const double *rates) {
    return guarded([&] {
        MK_REQUIRE(model, "null model");
        Model &m = *model->model;
        MK_REQUIRE(n_reactions >= 0 && n_reactions <= kMaxReactions, "0..16 reactions");
        if (n_reactions == 0) {
            m.R = 0;
            m.change.clear();
            m.rates.clear();
            return;
        }
        MK_REQUIRE(change && tuple_max && rates, "null argument");
        MK_REQUIRE(n_volume_classes >= 1 && (n_volume_classes == 1 || voxel_class),
                   "volume classes");
        m.R = n_reactions;
        m.change.assign(change, change + n_reactions * m.S);
        m.tmax.assign(tuple_max, tuple_max + m.S);
        for (int t : m.tmax) {
            MK_REQUIRE(t >= 0 && t <= 4096, "tuple bounds out of range");
        }
        m.nvc = n_volume_classes;
        m.vclass.clear();
        if (n_volume_classes > 1) {
            m.vclass.assign(voxel_class, voxel_class + m.V);
            for (int c : m.vclass) {
                MK_REQUIRE(c >= 0 && c < n_volume_classes, "volume class out of range");
            }
        }
        const int64_t total = static_cast<int64_t>(n_reactions) * n_volume_classes * m.ntuple();
        MK_REQUIRE(total < (int64_t(1) << 31), "rate table too large");
        m.rates.assign(rates, rates + total);
        m.validate();
    });
}

int mk_model_n_voxels(mk_model model, int64_t *n_voxels) {
    return guarded([&] {
        MK_REQUIRE(model && n_voxels, "null argument");
        *n_voxels = model->model->V;
    });
}

void mk_model_destroy(mk_model model) { delete model; }

// ---- generator

int mk_generator_create(mk_space space, mk_model model, int absorbing, mk_generator *out) {
    return guarded([&] {
        MK_REQUIRE(space && model && out, "null argument");
        auto h = std::make_unique<mk_generator_s>();
        const Space &sp = *space->space;
        h->space = Space::make(sp.V, sp.limits, sp.is_box);
        h->model = std::make_unique<Model>(*model->model);
        h->gen = std::make_unique<Generator>(*h->space, *h->model, absorbing != 0);
        *out = h.release();
    });
}

void mk_generator_destroy(mk_generator gen) { delete gen; }

int mk_generator_rows(mk_generator gen, int64_t *rows) {
    return guarded([&] {
        MK_REQUIRE(gen && rows, "null argument");
        *rows = gen->gen->op.n;
    });
}

int mk_generator_exit_leak(mk_generator gen, double *d_exit, double *d_leak, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && d_exit && d_leak, "null argument");
        gen->gen->apply<double>(kExitLeak, 0.0, nullptr, nullptr, d_exit, d_leak,
                                as_stream(stream));
    });
}

int mk_generator_n_jumps(mk_generator gen, int64_t *n_jumps, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && n_jumps, "null argument");
        *n_jumps = mkb::count_jumps(*gen->gen, as_stream(stream));
    });
}

int mk_generator_matrix(mk_generator gen, mk_csr *out, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && out, "null argument");
        auto m = std::make_unique<mk_csr_s>();
        mkb::assemble(*gen->gen, 0.0, 1.0, m->csr, as_stream(stream));
        *out = m.release();
    });
}

int mk_generator_characteristic_matrix(mk_generator gen, double shift, mk_csr *out, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && out, "null argument");
        MK_REQUIRE(std::isfinite(shift), "shift must be finite");
        auto m = std::make_unique<mk_csr_s>();
        mkb::assemble(*gen->gen, shift, -1.0, m->csr, as_stream(stream));
        *out = m.release();
    });
}

int mk_csr_size(mk_csr m, int64_t *rows, int64_t *nonzeros) {
    return guarded([&] {
        MK_REQUIRE(m && rows && nonzeros, "null argument");
        *rows = m->csr.rows;
        *nonzeros = m->csr.nnz;
    });
}

int mk_csr_device(mk_csr m, const int64_t **row_ptr, const int64_t **col, const double **val) {
    return guarded([&] {
        MK_REQUIRE(m && row_ptr && col && val, "null argument");
        *row_ptr = m->csr.row_ptr.get();
        *col = m->csr.col.get();
        *val = m->csr.val.get();
    });
}

int mk_csr_copy_host(mk_csr m, int64_t *row_ptr, int64_t *col, double *val) {
    return guarded([&] {
        MK_REQUIRE(m && row_ptr && (m->csr.nnz == 0 || (col && val)), "null argument");
        const auto &c = m->csr;
        check_cuda(cudaMemcpy(row_ptr, c.row_ptr.get(), sizeof(int64_t) * (c.rows + 1),
                              cudaMemcpyDeviceToHost),
                   "csr row_ptr copy");
        if (c.nnz > 0) {
            check_cuda(cudaMemcpy(col, c.col.get(), sizeof(int64_t) * c.nnz, cudaMemcpyDeviceToHost),
                       "csr col copy");
            check_cuda(cudaMemcpy(val, c.val.get(), sizeof(double) * c.nnz, cudaMemcpyDeviceToHost),
                       "csr val copy");
        }
    });
}

void mk_csr_destroy(mk_csr m) { delete m; }

int mk_generator_apply(mk_generator gen, const double *d_x, double *d_y, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && d_x && d_y, "null argument");
        gen->gen->apply<double>(kApplyQ, 0.0, d_x, nullptr, d_y, nullptr, as_stream(stream));
    });
}

int mk_generator_apply_shifted(mk_generator gen, double shift, const double *d_x, double *d_y,
                               void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && d_x && d_y, "null argument");
        gen->gen->apply<double>(kApplyShifted, shift, d_x, nullptr, d_y, nullptr,
                                as_stream(stream));
    });
}

int mk_generator_apply_shifted_batch(mk_generator gen, double shift, const double *d_x,
                                     double *d_y, int64_t ld, int nb, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && d_x && d_y, "null argument");
        MK_REQUIRE(nb >= 1 && nb <= kRowBatch, "batch must be in 1..4");
        MK_REQUIRE(ld >= gen->gen->op.n, "column stride shorter than the system");
        gen->gen->apply<double>(kApplyShifted, shift, d_x, nullptr, d_y, nullptr,
                                as_stream(stream), nb, ld);
    });
}

int mk_generator_apply_f32(mk_generator gen, const float *d_x, float *d_y, void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && d_x && d_y, "null argument");
        gen->gen->apply<float>(kApplyQ, 0.0f, d_x, nullptr, d_y, nullptr, as_stream(stream));
    });
}

int mk_generator_apply_shifted_f32(mk_generator gen, float shift, const float *d_x, float *d_y,
                                   void *stream) {
    return guarded([&] {
        MK_REQUIRE(gen && d_x && d_y, "null argument");
        gen->gen->apply<float>(kApplyShifted, shift, d_x, nullptr, d_y, nullptr,
                               as_stream(stream));
    });
}

// ---- multigrid

void mk_multigrid_options_default(mk_multigrid_options *opt) {
    if (!opt) {
        return;
    }
    const MultigridOptions d;
    opt->pre_sweeps = d.pre_sweeps;
    opt->post_sweeps = d.post_sweeps;
    opt->jacobi_weight = d.jacobi_weight;
    opt->coarsest_size = d.coarsest_size;
    opt->max_levels = d.max_levels;
    opt->coarse_cycles = d.coarse_cycles;
    opt->sweep_growth = d.sweep_growth;
    opt->smoother = d.smoother;
    opt->precision = d.precision;
    opt->batch = d.batch;
    opt->cycle_type = d.cycle_type;
}

static int fill_result(const SolverResult &r, mk_solver_result *out);

static MultigridOptions multigrid_options_of(const mk_multigrid_options *opt) {
    MultigridOptions o;
    if (opt) {
        MK_REQUIRE(opt->pre_sweeps >= 0 && opt->post_sweeps >= 0 && opt->coarse_cycles >= 1 &&
                       opt->sweep_growth >= 0 && opt->max_levels >= 1 && opt->coarsest_size >= 0,
                   "bad multigrid options");
        o.pre_sweeps = opt->pre_sweeps;
        o.post_sweeps = opt->post_sweeps;
        o.jacobi_weight = opt->jacobi_weight;
        o.coarsest_size = opt->coarsest_size;
        o.max_levels = opt->max_levels;
        o.coarse_cycles = opt->coarse_cycles;
        o.sweep_growth = opt->sweep_growth;
        o.smoother = opt->smoother;
        o.precision = opt->precision;
        o.batch = opt->batch;
        o.cycle_type = opt->cycle_type;
    }
    return o;
}

int mk_multigrid_create(mk_space space, mk_model model, double shift,
                        const mk_multigrid_options *opt, mk_multigrid *out) {
    return guarded([&] {
        MK_REQUIRE(space && model && out, "null argument");
        const MultigridOptions o = multigrid_options_of(opt);
        auto h = std::make_unique<mk_multigrid_s>();
        h->mg = std::make_unique<Multigrid>(*space->space, *model->model, shift, o);
        *out = h.release();
    });
}

int mk_multigrid_create_full(mk_space space, const mk_model *level_models, int n_levels, double shift,
                             const mk_multigrid_options *opt, mk_multigrid *out) {
    return guarded([&] {
        MK_REQUIRE(space && level_models && out && n_levels >= 1, "null argument");
        std::vector<const Model *> models;
        for (int d = 0; d < n_levels; ++d) {
            MK_REQUIRE(level_models[d], "null level model");
            models.push_back(level_models[d]->model.get());
        }
        const MultigridOptions o = multigrid_options_of(opt);
        auto h = std::make_unique<mk_multigrid_s>();
        h->mg = std::make_unique<Multigrid>(*space->space, models, shift, o);
        *out = h.release();
    });
}

int mk_multigrid_stationary(mk_multigrid mg, mk_generator gen, const double *d_b, double *d_x,
                            double tolerance, int64_t max_cycles, mk_solver_result *result,
                            void *stream) {
    SolverResult r;
    const int rc = guarded([&] {
        MK_REQUIRE(mg && gen && d_b && d_x, "null argument");
        MK_REQUIRE(tolerance >= 0.0 && max_cycles >= 0, "bad stationary-iteration options");
        r = stationary(*gen->gen, mg->mg->shift, *mg->mg, d_b, d_x, tolerance, max_cycles,
                       as_stream(stream));
    });
    if (rc != MK_OK) {
        return rc;
    }
    return fill_result(r, result);
}

void mk_multigrid_destroy(mk_multigrid mg) { delete mg; }

int mk_multigrid_apply(mk_multigrid mg, const double *d_b, double *d_x, void *stream) {
    return guarded([&] {
        MK_REQUIRE(mg && d_b && d_x, "null argument");
        mg->mg->apply(d_b, d_x, as_stream(stream));
    });
}

int mk_multigrid_apply_batch(mk_multigrid mg, const double *d_b, int64_t ldb, double *d_x,
                             int64_t ldx, int nb, void *stream) {
    return guarded([&] {
        MK_REQUIRE(mg && d_b && d_x, "null argument");
        MK_REQUIRE(ldb >= mg->mg->n && ldx >= mg->mg->n, "column stride shorter than the system");
        mg->mg->apply_batch(d_b, ldb, d_x, ldx, nb, as_stream(stream));
    });
}

int mk_multigrid_max_levels(mk_multigrid mg, int *levels) {
    return guarded([&] {
        MK_REQUIRE(mg && levels, "null argument");
        int best = 0;
        const auto &L0 = *mg->mg->levels[0];
        for (int k : L0.box_sector) {
            best = std::max(best, mg->mg->levels_of_sector(k));
        }
        *levels = best;
    });
}

int mk_multigrid_depth(mk_multigrid mg, int *depth) {
    return guarded([&] {
        MK_REQUIRE(mg && depth, "null argument");
        *depth = mg->mg->n_levels();
    });
}

int mk_multigrid_level_size(mk_multigrid mg, int depth, int64_t *n) {
    return guarded([&] {
        MK_REQUIRE(mg && n, "null argument");
        MK_REQUIRE(depth >= 0 && depth < mg->mg->n_levels(), "no such level");
        *n = mg->mg->levels[depth]->op.n;
    });
}

int mk_multigrid_restrict(mk_multigrid mg, int depth, const double *d_fine, double *d_coarse,
                          void *stream) {
    return guarded([&] {
        MK_REQUIRE(mg && d_fine && d_coarse, "null argument");
        mg->mg->transfer(depth, 0, d_fine, d_coarse, as_stream(stream));
    });
}

int mk_multigrid_prolong(mk_multigrid mg, int depth, const double *d_coarse, double *d_fine,
                         void *stream) {
    return guarded([&] {
        MK_REQUIRE(mg && d_fine && d_coarse, "null argument");
        mg->mg->transfer(depth, 1, d_coarse, d_fine, as_stream(stream));
    });
}

int mk_multigrid_apply_system(mk_multigrid mg, int depth, const double *d_x, double *d_y,
                              void *stream) {
    return guarded([&] {
        MK_REQUIRE(mg && d_x && d_y, "null argument");
        mg->mg->apply_system(depth, d_x, d_y, as_stream(stream));
    });
}

int mk_multigrid_smooth(mk_multigrid mg, int depth, const double *d_b, double *d_x, void *stream) {
    return guarded([&] {
        MK_REQUIRE(mg && d_b && d_x, "null argument");
        mg->mg->smooth(depth, d_b, d_x, as_stream(stream));
    });
}

// ---- GMRES

void mk_gmres_options_default(mk_gmres_options *opt) {
    if (!opt) {
        return;
    }
    const GmresOptions d;
    opt->tolerance = d.tolerance;
    opt->max_iterations = d.max_iterations;
    opt->restart = d.restart;
    opt->flexible = d.flexible;
}

static int create_solver(mk_generator gen, double shift, mk_multigrid mg, mk_precond pc,
                         const mk_gmres_options *opt, mk_solver *out) {
    return guarded([&] {
        MK_REQUIRE(gen && out, "null argument");
        auto h = std::make_unique<mk_solver_s>();
        h->gen = gen;
        h->mg = mg;
        h->pc = pc;
        h->shift = shift;
        if (opt) {
            MK_REQUIRE(opt->restart >= 1 && opt->max_iterations >= 0 && opt->tolerance >= 0.0,
                       "bad GMRES options");
            h->opt.tolerance = opt->tolerance;
            h->opt.max_iterations = opt->max_iterations;
            h->opt.restart = opt->restart;
            h->opt.flexible = opt->flexible;
        }
        const Preconditioner *M = preconditioner_of(*h);
        const bool flexible = h->opt.flexible || (M && M->varies());
        const int64_t n = gen->gen->op.n;
        MK_REQUIRE(!M || M->n == n, "preconditioner size does not match the system");
        const int m = static_cast<int>(std::min<int64_t>(h->opt.restart, std::max<int64_t>(n, 1)));
        h->ws = std::make_unique<Krylov>(n, m, flexible);
        *out = h.release();
    });
}

int mk_solver_create(mk_generator gen, double shift, mk_multigrid mg,
                     const mk_gmres_options *opt, mk_solver *out) {
    return create_solver(gen, shift, mg, nullptr, opt, out);
}

int mk_solver_create_pc(mk_generator gen, double shift, mk_precond pc,
                        const mk_gmres_options *opt, mk_solver *out) {
    return create_solver(gen, shift, nullptr, pc, opt, out);
}

void mk_solver_destroy(mk_solver solver) { delete solver; }

int mk_solver_set_tolerance(mk_solver solver, double tolerance) {
    return guarded([&] {
        MK_REQUIRE(solver, "null solver");
        MK_REQUIRE(tolerance >= 0.0, "tolerance must be nonnegative");
        solver->opt.tolerance = tolerance;
    });
}

static int fill_result(const SolverResult &r, mk_solver_result *out) {
    if (out) {
        out->iterations = r.iterations;
        out->residual = r.residual;
        out->converged = r.converged;
        out->status = r.status;
    }
    if (r.status == kENan) {
        return fail(MK_ENAN, "non-finite residual in GMRES");
    }
    if (r.status == kENotConv) {
        return fail(MK_ENOTCONV, "GMRES reached max_iterations");
    }
    return MK_OK;
}

int mk_solver_solve(mk_solver solver, const double *d_b, double *d_x, mk_solver_result *result,
                    void *stream) {
    SolverResult r;
    const int rc = guarded([&] {
        MK_REQUIRE(solver && d_b && d_x, "null argument");
        r = gmres(*solver->gen->gen, solver->shift, preconditioner_of(*solver),
                  d_b, d_x, solver->opt, *solver->ws, as_stream(stream));
    });
    if (rc != MK_OK) {
        return rc;
    }
    return fill_result(r, result);
}

int mk_solver_time_steps(mk_solver solver, int integrator, int steps, double rel_tolerance,
                         double *d_p, mk_solver_result *results, void *stream) {
    int status = MK_OK;
    const int rc = guarded([&] {
        MK_REQUIRE(solver && d_p, "null argument");
        MK_REQUIRE(integrator == 0 || integrator == 1, "integrator must be 0 (backward Euler) or 1 (Crank-Nicolson)");
        MK_REQUIRE(steps >= 0, "steps must be non-negative");
        MK_REQUIRE(rel_tolerance > 0.0 && std::isfinite(rel_tolerance), "rel_tolerance must be positive");
        const Generator &A = *solver->gen->gen;
        const int64_t n = A.op.n;
        const double s = solver->shift;
        cudaStream_t st = as_stream(stream);
        if (solver->b.size() != static_cast<std::size_t>(n)) {
            solver->b.resize(n);
            solver->x.resize(n);
        }
        DeviceArray<double> tmp(static_cast<std::size_t>(n)), partials(kDotBlocks), norm2(1);
        double *rhs = solver->b.get(), *x = solver->x.get();
        const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(double);
        const int solves = steps + (integrator == 1 && steps > 0 ? 1 : 0);
        for (int k = 0; k < solves; ++k) {
            check_cuda(cudaMemsetAsync(rhs, 0, bytes, st), "rhs");
            if (integrator == 1 && k >= 2) {
                // rhs = 2 s p - (s I - Q) p
                check_cuda(cudaMemsetAsync(tmp.get(), 0, bytes, st), "rhs");
                check_cuda(axpy(2.0 * s, d_p, tmp.get(), n, st), "rhs");
                A.apply<double>(kResidual, s, d_p, tmp.get(), rhs, nullptr, st);
            } else {
                check_cuda(axpy(s, d_p, rhs, n, st), "rhs");
            }
            check_cuda(dot(rhs, rhs, n, partials.get(), norm2.get(), st), "norm");
            double nr2 = 0.0;
            check_cuda(cudaMemcpyAsync(&nr2, norm2.get(), sizeof nr2, cudaMemcpyDeviceToHost, st), "norm");
            check_cuda(cudaMemcpyAsync(x, d_p, bytes, cudaMemcpyDeviceToDevice, st), "guess");
            check_cuda(cudaStreamSynchronize(st), "sync");
            GmresOptions o = solver->opt;
            o.tolerance = rel_tolerance * std::sqrt(nr2);
            const SolverResult r = gmres(A, s, preconditioner_of(*solver), rhs, x,
                                         o, *solver->ws, st);
            check_cuda(cudaMemcpyAsync(d_p, x, bytes, cudaMemcpyDeviceToDevice, st), "step");
            check_cuda(cudaStreamSynchronize(st), "sync");
            status = fill_result(r, results ? results + k : nullptr);
            if (status != MK_OK) {
                return;
            }
        }
    });
    return rc != MK_OK ? rc : status;
}

int mk_solver_solve_host(mk_solver solver, const double *h_b, double *h_x,
                         mk_solver_result *result, void *stream) {
    SolverResult r;
    const int rc = guarded([&] {
        MK_REQUIRE(solver && h_b && h_x, "null argument");
        const int64_t n = solver->gen->gen->op.n;
        if (solver->b.size() != static_cast<std::size_t>(n)) {
            solver->b.resize(n);
            solver->x.resize(n);
        }
        cudaStream_t s = as_stream(stream);
        const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(double);
        check_cuda(cudaMemcpyAsync(solver->b.get(), h_b, bytes, cudaMemcpyHostToDevice, s), "h2d");
        check_cuda(cudaMemcpyAsync(solver->x.get(), h_x, bytes, cudaMemcpyHostToDevice, s), "h2d");
        r = gmres(*solver->gen->gen, solver->shift, preconditioner_of(*solver),
                  solver->b.get(), solver->x.get(), solver->opt, *solver->ws, s);
        check_cuda(cudaMemcpyAsync(h_x, solver->x.get(), bytes, cudaMemcpyDeviceToHost, s), "d2h");
        check_cuda(cudaStreamSynchronize(s), "sync");
    });
    if (rc != MK_OK) {
        return rc;
    }
    return fill_result(r, result);
}

// ---- batched FGMRES

int mk_batch_solver_create(mk_generator gen, double shift, mk_multigrid mg,
                           const mk_gmres_options *opt, int width, mk_batch_solver *out) {
    return guarded([&] {
        MK_REQUIRE(gen && mg && out, "null argument");
        MK_REQUIRE(shift > 0.0, "shift must be positive");
        MK_REQUIRE(width >= 1 && width <= kRowBatch, "batch width must be in 1..4");
        MK_REQUIRE(mg->mg->opt.batch >= width, "the multigrid was built for a narrower batch");
        MK_REQUIRE(mg->mg->n == gen->gen->op.n, "multigrid and generator sizes differ");
        auto h = std::make_unique<mk_batch_solver_s>();
        h->gen = gen;
        h->mg = mg;
        h->shift = shift;
        if (opt) {
            MK_REQUIRE(opt->restart >= 1 && opt->max_iterations >= 0, "bad GMRES options");
            h->opt.max_iterations = opt->max_iterations;
            h->opt.restart = opt->restart;
        }
        h->opt.flexible = 1;
        const int64_t n = gen->gen->op.n;
        const int m = static_cast<int>(std::min<int64_t>(h->opt.restart, std::max<int64_t>(n, 1)));
        h->ws = std::make_unique<KrylovBatch>(n, m, width);
        h->b.resize(static_cast<std::size_t>(h->ws->ld) * width);
        h->x.resize(static_cast<std::size_t>(h->ws->ld) * width);
        *out = h.release();
    });
}

void mk_batch_solver_destroy(mk_batch_solver solver) { delete solver; }

int mk_batch_solver_solve(mk_batch_solver solver, const double *d_b, double *d_x, int64_t ld,
                          int nb, const double *h_tolerances, mk_solver_result *results,
                          void *stream) {
    std::vector<SolverResult> r;
    const int rc = guarded([&] {
        MK_REQUIRE(solver && d_b && d_x && h_tolerances && results, "null argument");
        KrylovBatch &ws = *solver->ws;
        MK_REQUIRE(nb >= 1 && nb <= ws.nb, "more columns than the solver's width");
        const int64_t n = ws.n;
        MK_REQUIRE(ld >= n, "column stride shorter than the system");
        cudaStream_t s = as_stream(stream);
        // columns into the workspace's stride, solve, and back
        for (int c = 0; c < nb; ++c) {
            check_cuda(cudaMemcpyAsync(solver->b.get() + c * ws.ld, d_b + c * ld, n * sizeof(double),
                                       cudaMemcpyDeviceToDevice, s),
                       "copy");
            check_cuda(cudaMemcpyAsync(solver->x.get() + c * ws.ld, d_x + c * ld, n * sizeof(double),
                                       cudaMemcpyDeviceToDevice, s),
                       "copy");
        }
        r = gmres_batch(*solver->gen->gen, solver->shift, *solver->mg->mg, solver->b.get(),
                        solver->x.get(), nb, h_tolerances, solver->opt, ws, s);
        for (int c = 0; c < nb; ++c) {
            check_cuda(cudaMemcpyAsync(d_x + c * ld, solver->x.get() + c * ws.ld, n * sizeof(double),
                                       cudaMemcpyDeviceToDevice, s),
                       "copy");
        }
    });
    if (rc != MK_OK) {
        return rc;
    }
    int first = MK_OK;
    for (int c = 0; c < nb; ++c) {
        const int st = fill_result(r[c], results + c);
        if (st != MK_OK && first == MK_OK) {
            first = st;
        }
    }
    return first;
}

} // extern "C"
