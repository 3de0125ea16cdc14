/* markovkit_b200 — C ABI of the B200 resolvent / FSP engine.
 *
 * Plain pointers and sizes only. Vectors named d_* are device pointers (the caller owns
 * them); h_* are host pointers. `stream` is a cudaStream_t passed as void* (NULL = the
 * default stream). Every call returns an MK_* status; mk_last_error() describes the last
 * failure on the calling thread. Handles own their device memory; *_destroy frees it.
 * A generator and a multigrid only read the space and model they were created from, and
 * copy what they need, so those may be destroyed afterwards.
 *
 * Each entry point names the MarkovKit interface it replaces (file:line in the reference).
 */
#ifndef MARKOVKIT_B200_H
#define MARKOVKIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* status codes; the C++ facade maps them back to the reference's exception types */
#define MK_OK 0
#define MK_EINVAL 1     /* std::invalid_argument */
#define MK_EOVERFLOW 2  /* std::overflow_error ("population state space is too large") */
#define MK_ESINGULAR 3  /* std::runtime_error ("singular block") */
#define MK_ENOMEM 4     /* device allocation failed */
#define MK_ENOTCONV 5   /* solver stopped at max_iterations (result still returned) */
#define MK_ENAN 6       /* non-finite residual */
#define MK_ETIMEOUT 7   /* a bounded wait gave up (mk_server_wait_for) */
#define MK_ECUDA 8      /* any other CUDA error */
#define MK_ETOLERANCE 9 /* std::runtime_error ("expv: the requested tolerance is too high") */
#define MK_ECANCELED 10 /* a queued server request was cancelled */

typedef struct mk_space_s *mk_space;
typedef struct mk_model_s *mk_model;
typedef struct mk_generator_s *mk_generator;
typedef struct mk_multigrid_s *mk_multigrid;
typedef struct mk_solver_s *mk_solver;

const char *mk_last_error(void);
int mk_version(void);
/* kernels this library has launched in this process (a graph launch counts its kernel nodes) */
int mk_kernel_launches(uint64_t *count);

/* Which kernel runs the rows of the solve passes (no reference counterpart; the reference has one
 * CPU code path): 0 (default) the stencil row kernel on the light rows of structured-grid levels
 * whose states hold one species of at most four molecules or two species of at most one (and
 * the pair-strip kernel, a block per pair of triangle rows, on the sectors of every pair of
 * voxels of one species), the general row kernel elsewhere; 1 the general kernel everywhere;
 * 2 as 0 without the pair-strip kernel. 0 and 2 give bit-identical results; 1 agrees with them
 * bit for bit on the stencil forms and to rounding on the pair forms (their exit terms add in
 * another order). The switch exists so that the paths can be compared. Process-wide; MK_EINVAL
 * for other values. */
int mk_set_row_path(int path);

/* ---- device memory helpers (for callers without their own CUDA runtime) ---- */
int mk_device_alloc(size_t bytes, void **d_ptr);
int mk_device_free(void *d_ptr);
int mk_memcpy_h2d(void *d_dst, const void *h_src, size_t bytes, void *stream);
int mk_memcpy_d2h(void *h_dst, const void *d_src, size_t bytes, void *stream);
int mk_stream_synchronize(void *stream);

/* ---- population state spaces: markovkit/rdme/population_space.hpp ---- */
/* population_box(n_voxels, max_totals)          population_space.hpp:131-139 */
int mk_space_create_box(int64_t n_voxels, int n_species, const int *max_totals, mk_space *out);
/* population_sector(n_voxels, totals)           population_space.hpp:105-109 */
int mk_space_create_sector(int64_t n_voxels, int n_species, const int *totals, mk_space *out);
void mk_space_destroy(mk_space space);
/* size(), n_sectors(), sector_begin(k), sector_totals(k)   population_space.hpp:141,156-159 */
int mk_space_size(mk_space space, int64_t *n);
int mk_space_n_sectors(mk_space space, int64_t *n_sectors);
int mk_space_sector_begin(mk_space space, int64_t k, int64_t *begin);
int mk_space_sector_totals(mk_space space, int64_t k, int *totals);
/* find_sector(totals) -> k or -1                population_space.hpp:166-175 */
int mk_space_find_sector(mk_space space, const int *totals, int64_t *k);
/* sector_of(i)                                  population_space.hpp:161-164 */
int mk_space_sector_of(mk_space space, int64_t i, int64_t *k);
/* find(x) -> index or -1, operator[](i) on one voxel-major state (host)
 *                                               population_space.hpp:142-150, :141 */
int mk_space_find_host(mk_space space, const int *h_state, int64_t *index);
int mk_space_state_host(mk_space space, int64_t i, int *h_state);
/* batched, on the device: d_states is count x (n_voxels * n_species) ints, voxel-major */
int mk_space_rank(mk_space space, const int *d_states, int64_t count, int64_t *d_index,
                  void *stream);
int mk_space_unrank(mk_space space, const int64_t *d_index, int64_t count, int *d_states,
                    void *stream);

/* ---- RDME models: markovkit/rdme/reaction_diffusion.hpp ---- */
/* voxel_domain(grid<D>(dims, spacing), diffusivities) reaction_diffusion.hpp:23-49,
 * with grid<D> = structured_grid_graph<D> (rdme/multigrid.hpp:20-21) */
int mk_model_create_grid(int dim, const int64_t *dims, const double *spacing, int n_species,
                         const double *diffusivities, mk_model *out);
/* voxel_domain(graph, volumes, diffusivities) with an explicit symmetric graph (CSR)
 *                                               reaction_diffusion.hpp:29-40 */
int mk_model_create_graph(int64_t n_voxels, const int64_t *nbr_ptr, const int64_t *nbr_idx,
                          const double *nbr_weight, const double *volumes, int n_species,
                          const double *diffusivities, mk_model *out);
/* the local reactions {change, rate(counts, volume)} of reaction_diffusion::reactions
 * (reaction_diffusion.hpp:62-67), tabulated by the caller: rates[r][c][tuple] is the rate of
 * reaction r in a voxel of volume class c whose counts n_s (0 <= n_s <= tuple_max[s]) have
 * tuple index sum_s n_s * prod_{s' > s} (tuple_max[s'] + 1). voxel_class may be NULL when
 * n_volume_classes == 1. */
int mk_model_set_reactions(mk_model model, int n_reactions, const int *change,
                           const int *tuple_max, int n_volume_classes, const int *voxel_class,
                           const double *rates);
int mk_model_n_voxels(mk_model model, int64_t *n_voxels);
void mk_model_destroy(mk_model model);

/* ---- the generator: markovkit/generator.hpp ---- */
/* generator(space, model, boundary)             generator.hpp:27-44; absorbing = 1 or 0 */
int mk_generator_create(mk_space space, mk_model model, int absorbing, mk_generator *out);
void mk_generator_destroy(mk_generator gen);
int mk_generator_rows(mk_generator gen, int64_t *rows);
/* exit_rates(), leak_rates()                    generator.hpp:55-59 */
int mk_generator_exit_leak(mk_generator gen, double *d_exit, double *d_leak, void *stream);
/* apply: y = Q x                                generator.hpp:62-70 */
int mk_generator_apply(mk_generator gen, const double *d_x, double *d_y, void *stream);
/* apply_shifted: y = shift x - Q x              generator.hpp:73-81 */
int mk_generator_apply_shifted(mk_generator gen, double shift, const double *d_x, double *d_y,
                               void *stream);
/* apply_shifted on nb <= 4 vectors at once (column c of x and y at c * ld): the row work is
 * done once for every column */
int mk_generator_apply_shifted_batch(mk_generator gen, double shift, const double *d_x,
                                     double *d_y, int64_t ld, int nb, void *stream);
int mk_generator_apply_f32(mk_generator gen, const float *d_x, float *d_y, void *stream);
int mk_generator_apply_shifted_f32(mk_generator gen, float shift, const float *d_x, float *d_y,
                                   void *stream);
/* n_jumps(): the jumps between states of the space     generator.hpp:48 */
int mk_generator_n_jumps(mk_generator gen, int64_t *n_jumps, void *stream);
/* generator::jumps(j) (markovkit/generator.hpp:50-53): the jumps out of state j that stay in
 * the space, as (to, rate) in the reference's order (diffusion by voxel, edge, species; then
 * reactions by voxel and reaction). Computed on the host from the generator's model. *count is
 * the number of jumps; the first min(count, capacity) are written (capacity 0 with NULL arrays
 * asks for the count). */
int mk_generator_jumps(mk_generator gen, int64_t j, int64_t *h_to, double *h_rate,
                       int64_t capacity, int64_t *count);

/* ---- the assembled generator: generator.hpp:84-107 ----
 * A CSR matrix in device memory owned by the handle: row_ptr[rows + 1], col[nonzeros] and
 * val[nonzeros], 64-bit indices, each row's columns ascending, the rates of distinct jumps
 * between one pair of states summed into one entry (num::spmat::from_triplets). Assembly
 * allocates device memory of about 40 bytes per entry while it runs; more than 2^31 - 1
 * entries before merging fails with MK_EOVERFLOW. */
typedef struct mk_csr_s *mk_csr;
/* matrix(): Q                                   generator.hpp:84 */
int mk_generator_matrix(mk_generator gen, mk_csr *out, void *stream);
/* characteristic_matrix(shift): shift I - Q     generator.hpp:87-90; shifted_generator::matrix()
 * generator.hpp:128 */
int mk_generator_characteristic_matrix(mk_generator gen, double shift, mk_csr *out, void *stream);
int mk_csr_size(mk_csr m, int64_t *rows, int64_t *nonzeros);
/* the device arrays (valid until mk_csr_destroy) */
int mk_csr_device(mk_csr m, const int64_t **row_ptr, const int64_t **col, const double **val);
/* copies into host arrays of rows + 1, nonzeros and nonzeros elements */
int mk_csr_copy_host(mk_csr m, int64_t *row_ptr, int64_t *col, double *val);
void mk_csr_destroy(mk_csr m);
/* a caller-given CSR matrix (host arrays, columns in range; duplicates are summed) on the device,
 * e.g. the generator of an explicit state list such as an FSP support (generator.hpp:27-44) */
int mk_csr_create_host(int64_t rows, const int64_t *row_ptr, const int64_t *col, const double *val,
                       mk_csr *out);
/* y = shift x + sign A x on device vectors (a warp per row): A x with (0, 1), s x - A x with (s, -1) */
int mk_csr_apply(mk_csr m, double shift, double sign, const double *d_x, double *d_y, void *stream);

/* ---- sector multigrid: markovkit/rdme/multigrid.hpp ---- */
typedef struct {
    int pre_sweeps;       /* multigrid_options, multigrid.hpp:125-134 */
    int post_sweeps;
    double jacobi_weight;
    int64_t coarsest_size;
    int max_levels;
    int coarse_cycles;
    int sweep_growth;
    int smoother;  /* 0 weighted Jacobi (reference default), 1 red-black Gauss-Seidel,
                      2 red-black ILU(0) (block ILU of rdme_full_multigrid.cpp:204-296 in colour order),
                      3 aggregate blocks (relaxation::aggregate_block, multigrid.hpp:239-341; batch 1) */
    int precision; /* 0 FP64, 1 FP32 (use inside flexible GMRES) */
    int batch;     /* right-hand sides one cycle can serve at once (1..4), for batch solvers */
    int cycle_type; /* 0 V or W (coarse_cycles); 1 K-cycle of the full-operator multigrid
                       (rdme_full_multigrid.cpp:851-878; FP64, batch 1; a nonlinear cycle:
                       flexible GMRES when used as a preconditioner) */
} mk_multigrid_options;
void mk_multigrid_options_default(mk_multigrid_options *opt);
/* sector_multigrid(domain, box, shift, options) multigrid.hpp:377-384; a single-sector
 * space gives population_multigrid (multigrid.hpp:145-179) */
int mk_multigrid_create(mk_space space, mk_model model, double shift,
                        const mk_multigrid_options *opt, mk_multigrid *out);
void mk_multigrid_destroy(mk_multigrid mg);
/* apply(b, x): one cycle per sector             multigrid.hpp:397-403 */
int mk_multigrid_apply(mk_multigrid mg, const double *d_b, double *d_x, void *stream);
/* the same cycle for nb <= options.batch right-hand sides at once (column c of b at
 * c * ldb, of x at c * ldx) */
int mk_multigrid_apply_batch(mk_multigrid mg, const double *d_b, int64_t ldb, double *d_x,
                             int64_t ldx, int nb, void *stream);
/* The same cycle for callers that must not allocate device memory during the call: a host that
 * fixes its device-memory budget at start-up and forbids allocation inside its compute
 * callbacks (a serving process that owns all of a GPU's memory, or a solver embedded in another
 * framework whose allocator it may not bypass). This entry point has no counterpart in the
 * reference. It calls no cudaMalloc or cudaFree: the work vectors of every level live in one
 * static device array of 64 MiB, which every GPU that loads the library holds until the process
 * exits. A hierarchy whose work vectors need more than that is rejected with MK_EINVAL and a
 * message giving the size. The first call on each device looks the array's address up
 * (cudaGetSymbolAddress) and caches it for the life of the process, so do not reset the device
 * (cudaDeviceReset) while the library is loaded. All calls share the one array and each overwrites it; calls that overlap on the GPU
 * (different streams, or different hierarchies at once) race and give wrong results, so order
 * them on one stream. Use a hierarchy from one host thread at a time, as with every mk_multigrid
 * call. The result equals mk_multigrid_apply's bit for bit. */
int mk_multigrid_apply_noalloc(mk_multigrid mg, const double *d_b, double *d_x, void *stream);
/* max_levels()                                  multigrid.hpp:389-395 */
int mk_multigrid_max_levels(mk_multigrid mg, int *levels);
int mk_multigrid_depth(mk_multigrid mg, int *depth);
int mk_multigrid_level_size(mk_multigrid mg, int depth, int64_t *n);
/* population_transfer restrict / prolong between depth d and d+1 (multigrid.hpp:100-111)
 * and apply_system at depth d (multigrid.hpp:196), FP64 */
int mk_multigrid_restrict(mk_multigrid mg, int depth, const double *d_fine, double *d_coarse,
                          void *stream);
int mk_multigrid_prolong(mk_multigrid mg, int depth, const double *d_coarse, double *d_fine,
                         void *stream);
int mk_multigrid_apply_system(mk_multigrid mg, int depth, const double *d_x, double *d_y,
                              void *stream);
/* one sweep of the level's smoother on (b, x) at depth d, in place on x (FP64 hierarchies):
 * the weighted Jacobi update of population_multigrid::smooth (multigrid.hpp:309-317), a
 * red-then-black Gauss-Seidel pass pair, or one red-black ILU(0) sweep x += (LU)^-1 (b - A x) */
int mk_multigrid_smooth(mk_multigrid mg, int depth, const double *d_b, double *d_x, void *stream);

/* ---- GMRES: num::gmres(A, [M], b, x, options) (call sites tests/test_rdme.cpp:238-249) ---- */
typedef struct {
    double tolerance;       /* absolute, on ||b - A x||_2 */
    int64_t max_iterations; /* Arnoldi steps in total */
    int restart;
    int flexible;           /* FGMRES; forced on with an FP32 preconditioner */
} mk_gmres_options;
typedef struct {
    int64_t iterations;
    double residual; /* recomputed true residual norm */
    int converged;
    int status;
} mk_solver_result;
void mk_gmres_options_default(mk_gmres_options *opt);
/* The full-operator multigrid of the paper driver (rdme/cpp/rdme_full_multigrid.cpp:348-560,
 * 819-850; no counterpart in the library): every level is the whole box on the grid coarsened
 * d times, with the diffusivities doubled per level and the reactions of level_models[d],
 * tabulated by the caller at that level's voxel volume (level_models[0] is the fine model; the
 * grids must be those coarsen() gives). Transfers as sector_multigrid's; the level where the grid
 * stops coarsening (or n_levels is reached) is inverted densely as one block (at most 8192
 * states). Smoother 0 (weighted Jacobi) only; coarse_cycles 2 gives the W-cycle. Use it as a
 * GMRES preconditioner (mk_solver_create) or as a solver of its own: */
int mk_multigrid_create_full(mk_space space, const mk_model *level_models, int n_levels, double shift,
                             const mk_multigrid_options *opt, mk_multigrid *out);
/* the stationary iteration x <- x + M (b - A x), A = shift I - Q of gen with the multigrid's
 * shift, from the x given, until ||b - A x||_2 <= tolerance (MK_ENOTCONV after max_cycles);
 * result->iterations counts the cycles */
int mk_multigrid_stationary(mk_multigrid mg, mk_generator gen, const double *d_b, double *d_x,
                            double tolerance, int64_t max_cycles, mk_solver_result *result,
                            void *stream);

/* a resident solver for A = shift I - Q (shifted_generator, generator.hpp:116-133),
 * preconditioned by mg (NULL: plain GMRES); it keeps the Krylov workspace on the device */
int mk_solver_create(mk_generator gen, double shift, mk_multigrid mg,
                     const mk_gmres_options *opt, mk_solver *out);
void mk_solver_destroy(mk_solver solver);
/* change the absolute tolerance of a resident solver (e.g. 1e-10 * ||b|| per right-hand side) */
int mk_solver_set_tolerance(mk_solver solver, double tolerance);
/* x is the initial guess on entry and the solution on return (device vectors) */
int mk_solver_solve(mk_solver solver, const double *d_b, double *d_x, mk_solver_result *result,
                    void *stream);
/* the same with host vectors: copies in, solves, copies out */
int mk_solver_solve_host(mk_solver solver, const double *h_b, double *h_x,
                         mk_solver_result *result, void *stream);
/* Time stepping by repeated resolvents (no counterpart in the library; the paper driver's
 * integrators, rdme/cpp/rdme_full_multigrid.cpp:1173-1238), on the device vector d_p of the
 * solver's size, in place. With the solver's shift s:
 *   integrator 0, backward Euler: p <- (s I - Q)^{-1} (s p), one step of length 1/s;
 *   integrator 1, Crank-Nicolson with a Rannacher start (s = 2/dt): two backward-Euler steps of
 *     length dt/2, then p <- (s I - Q)^{-1} (2 s p - (s I - Q) p) per step of length dt;
 *     `steps` counts the steps of length dt, so steps + 1 solves run.
 * Each solve starts from the current p and stops at ||rhs - A p|| <= rel_tolerance * ||rhs||;
 * results[k] (optional, steps + integrator entries) reports solve k. Stops at the first solve
 * that does not converge and returns its status. */
int mk_solver_time_steps(mk_solver solver, int integrator, int steps, double rel_tolerance,
                         double *d_p, mk_solver_result *results, void *stream);

/* ---- Preconditioners: the right preconditioner M of num::gmres(A, M, b, x, options) as any
 * operator, not only a multigrid (examples/rdme_multigrid_benchmark.cpp:82-115):
 *   diagonal   num::jacobi_preconditioner(inverse_diagonal): z = d .* v
 *   ilu0       num::ilu0_preconditioner(A): ILU(0) of a CSR matrix in its natural row order,
 *              factored on the device over level sets of rows (Saad, Alg. 10.4), applied as
 *              level-scheduled triangular solves
 *   multigrid  a sector multigrid as a preconditioner handle
 *   host       any other operator: z = fn(ctx, v) on the host, v and z host arrays of n
 * A solver made with mk_solver_create_pc uses flexible GMRES when the preconditioner varies
 * (an FP32 multigrid). The handle must outlive the solvers that use it. ---- */
typedef struct mk_precond_s *mk_precond;
typedef int (*mk_precond_host_fn)(void *ctx, const double *v, double *z, int64_t n);
int mk_precond_create_diagonal(int64_t n, const double *h_inverse_diagonal, mk_precond *out);
/* row_ptr[n + 1]; each row's columns strictly ascending with the diagonal present (MK_EINVAL
 * otherwise); MK_ESINGULAR on a zero or non-finite pivot */
int mk_precond_create_ilu0(int64_t n, const int64_t *h_row_ptr, const int64_t *h_col,
                           const double *h_val, void *stream, mk_precond *out);
int mk_precond_create_multigrid(mk_space space, mk_model model, double shift,
                                const mk_multigrid_options *opt, mk_precond *out);
/* fn returns 0 on success; anything else fails the solve with MK_EINVAL */
int mk_precond_create_host(int64_t n, mk_precond_host_fn fn, void *ctx, mk_precond *out);
void mk_precond_destroy(mk_precond pc);
int mk_precond_size(mk_precond pc, int64_t *n);
/* z = M v on device vectors */
int mk_precond_apply(mk_precond pc, const double *d_v, double *d_z, void *stream);
/* an ILU(0) preconditioner's level sets: depth of the forward and backward sweeps, and the
 * kernel launches one application takes (runs of thin levels share a launch) */
int mk_precond_ilu0_schedule(mk_precond pc, int64_t *lower_levels, int64_t *upper_levels,
                             int64_t *launches_per_apply);
/* a resident solver for shift I - Q preconditioned by pc (NULL: plain GMRES) */
int mk_solver_create_pc(mk_generator gen, double shift, mk_precond pc,
                        const mk_gmres_options *opt, mk_solver *out);

/* Several resolvent solves of one system at once (no counterpart in the reference; each column
 * is num::gmres(A, M, b, x)): flexible GMRES advancing up to `width` right-hand sides in
 * lockstep, one batched operator apply and one batched multigrid cycle per step for all of
 * them. mg must have been created with options.batch >= width. */
typedef struct mk_batch_solver_s *mk_batch_solver;
int mk_batch_solver_create(mk_generator gen, double shift, mk_multigrid mg,
                           const mk_gmres_options *opt, int width, mk_batch_solver *out);
void mk_batch_solver_destroy(mk_batch_solver solver);
/* nb <= width columns: column c of b and x at d_b + c * ld and d_x + c * ld (ld >= rows);
 * x holds the initial guesses; column c stops at the absolute tolerance h_tolerances[c];
 * results[c] per column. Returns the first column's failing status, if any. */
int mk_batch_solver_solve(mk_batch_solver solver, const double *d_b, double *d_x, int64_t ld,
                          int nb, const double *h_tolerances, mk_solver_result *results,
                          void *stream);

/* ---- Krylov FSP: solve_krylov_fsp(model, initial, final_time, options), markovkit/fsp.hpp ---- */
/* krylov_fsp_options (fsp.hpp:190-202) with inside = box(bounds) (fsp.hpp:26-35); save_every
 * has no counterpart: only the final distribution is kept. method 1 runs solve_adaptive_fsp
 * instead (fsp.hpp:108-188) with adaptive_fsp_options' step_scale, prune_fraction,
 * flux_tolerance and min_probability (layers, max_steps (steps), krylov_dim and krylov_tol as
 * named; sampled_expansion is not offered) */
typedef struct {
    double tolerance;        /* the probability that may leak by final_time */
    double initial_step;
    double step_growth;
    double drop_probability;
    double drop_derivative;
    int layers;
    int krylov_dim;          /* 1..30 */
    int64_t max_steps;       /* attempts (method 1: steps) */
    double krylov_tol;
    int method;              /* 0 solve_krylov_fsp, 1 solve_adaptive_fsp */
    double step_scale;       /* method 1: each step expects about this many jumps */
    double prune_fraction;   /* method 1: the least likely fraction of states may be pruned ... */
    double flux_tolerance;   /* ... if its probability flux is below this share of the total */
    double min_probability;  /* method 1: also prune any state below this probability */
} mk_fsp_options;
void mk_fsp_options_default(mk_fsp_options *opt);
/* One instance. A reaction_network (markovkit/reaction_network.hpp:11-39) restricted to the
 * box 0 <= x_s <= bounds[s], with its propensities tabulated by the caller over the box:
 * rates[r * box_size + i] = rate of reaction r in the state with box index
 * i = sum_s x_s * prod_{s' > s} (bounds[s'] + 1) (species 0 most significant). Jumps with a
 * rate that is not > 0 do not exist, as in reaction_network::transitions. The initial state
 * (a delta, fsp.hpp:209) must lie in the box. */
typedef struct {
    int n_species;           /* 1..4 */
    int n_reactions;         /* 0..16 */
    const int *bounds;       /* n_species */
    const int *change;       /* n_reactions x n_species */
    const double *rates;     /* n_reactions x box_size, host memory */
    const int *initial;      /* n_species */
    double final_time;
    mk_fsp_options options;
} mk_fsp_problem;
typedef struct {
    double time;             /* fsp_solution::times.back() */
    int64_t attempts;
    int64_t accepted;
    int64_t support;         /* states in the final support */
    int64_t substeps;        /* expv time steps over all attempts */
    int64_t applies;         /* operator applies over all attempts */
    int status;              /* MK_OK, MK_ENOTCONV (stopped before final_time), MK_ETOLERANCE, MK_ENAN */
    int clipped;             /* bit s set when an expansion met a jump to a state above bounds[s]:
                                the box, not the network, kept that state out of the support */
} mk_fsp_result;
typedef struct mk_fsp_batch_s *mk_fsp_batch;
/* the number of states in box(bounds) */
int mk_fsp_box_size(int n_species, const int *bounds, int64_t *size);
/* Uploads n instances (their rate tables included) and sizes the workspace. The instances
 * run in one persistent kernel, largest box first, one thread block per instance at a time. */
int mk_fsp_batch_create(int n, const mk_fsp_problem *problems, mk_fsp_batch *out);
void mk_fsp_batch_destroy(mk_fsp_batch batch);
/* total states over all boxes (the length of the output) and, unless h_offsets is NULL, the
 * offset of each instance's box in it (n entries; instance k's box follows instance k-1's) */
int mk_fsp_batch_output_size(mk_fsp_batch batch, int64_t *total, int64_t *h_offsets);
/* block shape: threads per block (128, 256 or 512) and number of blocks (0 = all that fit) */
int mk_fsp_batch_set_shape(mk_fsp_batch batch, int threads, int blocks);
int mk_fsp_batch_get_shape(mk_fsp_batch batch, int *threads, int *blocks);
/* times every shape on `sample` evenly spaced instances (0 = all) and keeps the fastest */
int mk_fsp_batch_autotune(mk_fsp_batch batch, int sample, void *stream);
/* runs every instance; stream-ordered */
int mk_fsp_batch_run(mk_fsp_batch batch, void *stream);
/* the device array of final distributions (each over its box, in box order) */
int mk_fsp_batch_device_output(mk_fsp_batch batch, const double **d_out);
/* copies results and (unless h_out is NULL) the distributions to the host, synchronising the
 * stream; returns the first instance's failing status, with mk_last_error naming it */
int mk_fsp_batch_results(mk_fsp_batch batch, double *h_out, mk_fsp_result *results,
                         void *stream);
/* create, run, copy out, destroy: solve_krylov_fsp for each problem */
int mk_fsp_krylov_batch(int n, const mk_fsp_problem *problems, double *h_out,
                        mk_fsp_result *results, void *stream);

/* ---- Batched SSA: gillespie(model, x, final_time, random, max_jumps) and tau_leaping(model, x,
 * final_time, random, leap_options) (markovkit/ssa.hpp:42-113), `paths` independent paths in one
 * launch, one per thread. The network is described as for mk_fsp_problem: propensities
 * tabulated over the box 0 <= x_s <= bounds[s]; a transition exists when its rate is > 0 and
 * its result has no negative count (reaction_network::transitions). A path whose next state
 * would leave the box stops there with status MK_EOVERFLOW (mk_ssa_run then returns
 * MK_EOVERFLOW): widen the box and run again; path i is a function of (seed, i) alone, so a
 * rerun replays it exactly. Random numbers: Philox4x32-10 keyed by the seed (the reference
 * draws from a host generator, so paths agree with it in distribution, not sample by sample).
 * Per path the outputs hold the final state, the state at each observation time (the state
 * occupied at t, trajectory::indices_at), the jumps (or leaps) taken and a status, and when
 * record > 0 the first `record` entries (times, states) of the path as the reference's
 * trajectory holds them, with the full count. ---- */
typedef struct {
    int n_species;                  /* 1..4 */
    int n_reactions;                /* 0..16 */
    const int *bounds;              /* n_species */
    const int *change;              /* n_reactions x n_species */
    const double *rates;            /* n_reactions x box_size, host memory (as mk_fsp_problem) */
    const int *initial;             /* n_species, inside the box */
    double final_time;
    int method;                     /* 0 Gillespie's direct method, 1 Poisson tau-leaping */
    int64_t max_jumps;              /* Gillespie: jumps per path (ssa.hpp:44) */
    double leap_step;               /* tau-leaping leap_options: step (0: from epsilon), */
    double leap_epsilon;            /* epsilon and */
    double leap_min_step;           /* min_step (ssa.hpp:77-81) */
    int64_t paths;
    uint64_t seed;
    int n_observations;
    const double *observation_times; /* sorted, within [0, final_time] */
    int record;                     /* trajectory entries kept per path; 0: none */
} mk_ssa_problem;
typedef struct {                    /* host arrays; observed and record_* may be NULL when unused */
    int *final_state;               /* paths x n_species */
    int *observed;                  /* paths x n_observations x n_species */
    int64_t *steps;                 /* paths: jumps (Gillespie) or leaps (tau-leaping) */
    int *status;                    /* paths: MK_OK, MK_EOVERFLOW (left the box), MK_ENOTCONV */
    double *record_times;           /* paths x record */
    int *record_states;             /* paths x record x n_species */
    int *record_count;              /* paths: entries of the whole trajectory */
} mk_ssa_output;
/* defaults: max_jumps unlimited, leap_epsilon 0.03, leap_min_step 1e-6, one path */
void mk_ssa_problem_default(mk_ssa_problem *problem);
int mk_ssa_run(const mk_ssa_problem *problem, mk_ssa_output *out, void *stream);

/* ---- Serving: a request loop of resolvent solves (no counterpart in the reference; each
 * request is the reference's shifted_generator + sector_multigrid + num::gmres solve,
 * tests/test_rdme.cpp:225-251, on a resident solver) ----
 * Requests are served first come, first served by `slots` worker threads, each with its own
 * CUDA stream, so up to `slots` solves overlap on the device. A resident solver (generator,
 * multigrid, Krylov workspace) is kept per (problem, shift) for later requests. New solvers are
 * admitted by their HBM footprint against the budget: idle solvers are evicted least recently
 * used first, and a worker waits while the rest are busy. h_b and h_x are host arrays of the
 * problem's size that must stay valid until the request completes. */
typedef struct {
    int slots;               /* concurrent solves (worker threads and streams), 1..64 */
    size_t hbm_budget;       /* bytes for resident solvers; 0 = 80 % of the free memory */
    int precision;           /* 1: FP32 multigrid inside FP64 flexible GMRES; 0: all FP64 */
    int smoother;            /* multigrid smoother: 0 Jacobi, 1 red-black Gauss-Seidel, 2 ILU(0);
                              * -1 per problem: Gauss-Seidel for one species of at most two
                              * molecules per state, Jacobi otherwise */
    int restart;             /* GMRES restart, 1..64 */
    int64_t max_iterations;
    double rel_tolerance;    /* stop at ||b - A x|| <= rel_tolerance * ||b|| */
    int batch;               /* queued requests with the same problem and shift solved together
                              * by one batched FGMRES, 1..4: a problem's resident solvers are the
                              * widest up to this whose footprint is at most hbm_budget / slots,
                              * else one request wide */
    int64_t coarsest_size;   /* multigrid sectors of at most this many states get a dense solve */
} mk_server_options;
typedef struct {
    int64_t ticket;
    int status;              /* MK_OK, MK_ENOTCONV, MK_ENOMEM (footprint above the budget), ... */
    int64_t iterations;
    double residual;         /* relative true residual */
    double latency_ms;       /* submit to x on the host */
    double queue_ms;         /* submit to having a slot and the memory */
    double solve_ms;         /* the rest: set-up of a new resident solver, copies, solve */
    int batched;             /* requests solved together with this one (itself included) */
} mk_server_result;
typedef struct {
    int64_t completed;
    double p50_ms, p99_ms;   /* latency percentiles over completed requests */
    double solves_per_s;     /* completed / (first submit .. last completion) */
    size_t resident_bytes, budget_bytes;
    int64_t resident_solvers, evictions, memory_waits;
} mk_server_stats;
typedef struct mk_server_s *mk_server;
void mk_server_options_default(mk_server_options *opt);
int mk_server_create(const mk_server_options *opt, mk_server *out);
/* finishes the queued requests, then stops the workers and frees every resident solver */
void mk_server_destroy(mk_server server);
/* copies what the server needs of a space and a model; returns the problem's number */
int mk_server_register(mk_server server, mk_space space, mk_model model, int *problem);
/* the footprint the admission control charges for a solver of this problem */
int mk_server_footprint(mk_server server, int problem, size_t *bytes);
int mk_server_submit(mk_server server, int problem, double shift, const double *h_b, double *h_x,
                     int64_t *ticket);
/* blocks until the request is done; returns its status */
int mk_server_wait(mk_server server, int64_t ticket, mk_server_result *result);
/* the same, giving up with MK_ETIMEOUT after timeout_ms (the request stays queued or running) */
int mk_server_wait_for(mk_server server, int64_t ticket, double timeout_ms,
                       mk_server_result *result);
/* removes a request that no worker has taken yet; its result then carries MK_ECANCELED.
 * MK_EINVAL when it has already started or finished. */
int mk_server_cancel(mk_server server, int64_t ticket);
/* blocks until every submitted request is done */
int mk_server_drain(mk_server server);
int mk_server_stats_get(mk_server server, mk_server_stats *stats);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* MARKOVKIT_B200_H */
