// Host side of the B200 resolvent engine: population spaces, RDME models, the matrix-free
// generator, the sector multigrid hierarchy and (flexible) GMRES. Everything here owns device
// memory and launches the sm_100a kernels of row_kernels.cu and krylov.cu on a caller stream.
#pragma once

#include "aggregate.cuh"
#include "host_model.hpp"
#include "krylov.cuh"
#include "launch_count.hpp"
#include "row_kernels.cuh"
#include "transfer.cuh"

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mkb {

void check_cuda(cudaError_t e, const char *what);

template <typename T>
class DeviceArray {
  public:
    DeviceArray() = default;
    explicit DeviceArray(std::size_t n) { resize(n); }
    ~DeviceArray() { release(); }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept : p_(o.p_), n_(o.n_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void resize(std::size_t n) {
        release();
        if (n > 0) {
            check_cuda(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)), "cudaMalloc");
            n_ = n;
        }
    }
    void upload(const std::vector<T> &h) {
        resize(h.size());
        if (!h.empty()) {
            check_cuda(cudaMemcpy(p_, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice),
                       "upload");
        }
    }
    [[nodiscard]] T *get() const { return p_; }
    [[nodiscard]] std::size_t size() const { return n_; }

  private:
    void release() {
        if (p_) {
            cudaFree(p_);
        }
        p_ = nullptr;
        n_ = 0;
    }
    T *p_ = nullptr;
    std::size_t n_ = 0;
};

// C(q, j), 0 <= j <= jmax, 0 <= q <= qmax, on host and device (saturating at 2^62)
struct Binomials {
    int jmax = 0, qmax = 0;
    std::vector<std::int64_t> host;
    DeviceArray<std::int64_t> dev;
    Binomials(int jmax_, int qmax_) : jmax(jmax_), qmax(qmax_), host(binomial_table(jmax_, qmax_)) {
        dev.upload(host);
    }
    [[nodiscard]] BinomTable host_view() const { return {host.data(), jmax, qmax}; }
    [[nodiscard]] BinomTable device_view() const { return {dev.get(), jmax, qmax}; }
};

constexpr int kHostIndexCap = 1024; // largest species total the host rank/unrank accept

// Every sector of a box (0 <= t_s <= max_s, mixed-radix order, species 0 most significant,
// markovkit/rdme/population_space.hpp:131-196) or a single sector (:105-127).
struct Space {
    int V = 0, S = 0;
    bool is_box = true;
    std::vector<int> limits; // box: max totals; sector: totals
    std::vector<SectorDesc> sectors;
    std::int64_t n = 0;
    int max_total = 0; // largest total of one species
    int max_mol = 0;   // largest molecules in one state
    std::shared_ptr<Binomials> binom;
    DeviceArray<SectorDesc> d_sectors;
    DeviceArray<int> d_limits;

    static std::unique_ptr<Space> make(int V, const std::vector<int> &limits, bool is_box);
    [[nodiscard]] int find_sector(const int *totals) const;
    [[nodiscard]] std::int64_t rank(const int *state) const; // -1: not in the space
    void unrank(std::int64_t i, int *state) const;
    [[nodiscard]] int sector_of(std::int64_t i) const;
};

// host + device tables of one voxel graph and model in one precision
template <typename T>
struct ModelTables {
    HostTables<T> h;
    DeviceArray<int> nbr_ptr, nbr_idx, vclass;
    DeviceArray<T> in_coef, deg_coef, rate;
    DeviceArray<unsigned char> vparity;
    DeviceArray<unsigned> vmask;
    ModelView<T> host, dev;
    void build(const Model &m, double diff_scale, bool with_reactions, bool absorbing);
};

// Which kernel runs the rows of the solve passes: 0 (default) the stencil kernel wherever a level
// allows it, 1 the general kernel everywhere (both give bit-identical results).
void set_row_path(int path);
int row_path();

// A level space with one model: the unit the row kernels run over.
struct OperatorLevel {
    int V = 0, S = 0;
    std::int64_t n = 0;
    int mol_cap = 4;
    std::vector<SectorDesc> sectors;
    DeviceArray<SectorDesc> d_sectors;
    std::vector<Tile> tiles; // every row
    DeviceArray<Tile> d_tiles;
    // the same rows split between the stencil kernel (light rows of a structured grid in a
    // stencil shape) and the general kernel (the rest); empty when the level has no stencil rows
    std::vector<Tile> stencil_tiles, general_tiles;
    DeviceArray<Tile> d_stencil_tiles, d_general_tiles;
    // rows with in-jumps from every voxel that the pair-form heavy kernel serves in the operator
    // passes (then general_rest holds the general kernel's other rows)
    std::vector<Tile> heavy_tiles, general_rest;
    DeviceArray<Tile> d_heavy_tiles, d_general_rest;
    // two-molecule sectors of one species in the pair-strip form (kind-3 tiles, a block per pair
    // of triangle rows) and the stencil kernel's other rows; empty when no sector qualifies
    std::vector<Tile> strip_tiles, stencil_rest;
    DeviceArray<Tile> d_strip_tiles, d_stencil_rest;
    // heavy rows of one molecule whose heavy sources are the pair sector, eight a block (kind-4
    // tiles); heavy_tiles then holds the other heavy rows
    std::vector<Tile> heavy_group_tiles;
    DeviceArray<Tile> d_heavy_group_tiles;
    // tables of the pair and single-molecule row forms (stencil_tables.hpp), per precision
    std::vector<StencilSector<double>> h_ss64;
    DeviceArray<StencilSector<double>> ss64;
    DeviceArray<StencilSector<float>> ss32;
    DeviceArray<double> ddeg64;
    DeviceArray<float> ddeg32;
    StencilView<double> sv64;
    StencilView<float> sv32;
    ModelTables<double> t64;
    ModelTables<float> t32;
    std::shared_ptr<Binomials> binom;

    // sector couplings (src/dst/heavy) for the model's reactions, then tiles and uploads
    void finalize(const Model &m, bool with_reactions);
    template <typename T>
    [[nodiscard]] RowParams<T> params() const;
    template <typename T>
    void run(RowMode mode, const RowParams<T> &p, cudaStream_t stream) const;
};

struct Generator {
    const Space *space = nullptr;
    OperatorLevel op;
    bool absorbing = true;
    std::int64_t n_jumps_cache = -1;
    Generator(const Space &space, const Model &model, bool absorbing);
    // one pass over every row; with nb > 1, nb right-hand sides whose columns sit ld apart
    template <typename T>
    void apply(RowMode mode, T shift, const T *x, const T *b, T *y, T *aux, cudaStream_t stream,
               int nb = 1, std::int64_t ld = 0) const;
};

struct MultigridOptions {
    int pre_sweeps = 2;
    int post_sweeps = 2;
    double jacobi_weight = 2.0 / 3.0;
    std::int64_t coarsest_size = 4;
    int max_levels = 32;
    int coarse_cycles = 1;
    int sweep_growth = 0;
    int smoother = 0;  // 0 weighted Jacobi (the reference's default), 1 red-black Gauss-Seidel,
                       // 2 red-black ILU(0), 3 aggregate blocks (relaxation::aggregate_block)
    int precision = 0; // 0 FP64, 1 FP32 preconditioner
    int batch = 1;     // right-hand sides one cycle can serve at once (work vectors per level)
    int cycle_type = 0; // 0 V/W cycles (coarse_cycles), 1 K-cycle (full-operator hierarchy, FP64)
};

// A right preconditioner z = M v of gmres(): FP64 in and out, device vectors of n entries,
// enqueued on `stream`. The reference takes any linear operator with apply(x, y) as num::gmres's
// preconditioner (examples/rdme_multigrid_benchmark.cpp:82-115): the multigrid below, the
// diagonal and ILU(0) ones of precond.cuh, or a host callback.
struct Preconditioner {
    std::int64_t n = 0;
    Preconditioner() = default;
    explicit Preconditioner(std::int64_t n_) : n(n_) {}
    virtual ~Preconditioner() = default;
    Preconditioner(const Preconditioner &) = delete;
    Preconditioner &operator=(const Preconditioner &) = delete;
    virtual void apply(const double *v, double *z, cudaStream_t stream) = 0;
    // true when M is not one fixed linear map (FP32 arithmetic inside): GMRES must then keep
    // the preconditioned basis (flexible GMRES)
    [[nodiscard]] virtual bool varies() const { return false; }
};

// sector_multigrid (markovkit/rdme/multigrid.hpp:136-408): one geometric V-cycle per
// population sector on the diffusion-only operator, all sectors of a depth in one launch.
struct Multigrid : Preconditioner {
    struct Level {
        OperatorLevel op;
        int pre = 2, post = 2;
        // transfer to the next level: parent voxels (set-up), and per fine state its coarse state
        // and prolongation weight; the fine states of each coarse state in ascending order
        DeviceArray<int> parent;
        DeviceArray<double> log_children;
        DeviceArray<int> coarse_of, children, child_begin;
        DeviceArray<double> w64;
        DeviceArray<float> w32;
        // dense terminal blocks of sectors that stop here
        std::vector<TerminalBlock> h_term;
        DeviceArray<TerminalBlock> d_term;
        DeviceArray<double> inv64;
        DeviceArray<float> inv32;
        // red-black ILU(0) pivots (smoother 2): diagonal on colour 0, modified on colour 1
        DeviceArray<double> piv64;
        DeviceArray<float> piv32;
        // aggregate-block smoother (smoother 3): the blocks of coarse voxel a are
        // [agg_ptr[a], agg_ptr[a + 1]); the terminal sectors keep Jacobi on their dense blocks
        std::vector<int> agg_ptr;
        DeviceArray<AggBlock> agg_blocks;
        DeviceArray<int> agg_states, agg_row_col;
        DeviceArray<std::int64_t> agg_row_ptr;
        DeviceArray<double> agg_val64, agg_inv64, agg_r64, agg_e64;
        DeviceArray<float> agg_val32, agg_inv32, agg_r32, agg_e32;
        std::vector<DenseBlock> h_dense;
        DeviceArray<DenseBlock> d_dense;
        DeviceArray<double> dense64;
        DeviceArray<float> dense32;
        // work vectors (precision of the preconditioner)
        DeviceArray<double> rhs64, x64, tmp64, r64, acc64, crhs64;
        DeviceArray<float> rhs32, x32, tmp32, r32, acc32, crhs32;
        std::vector<int> box_sector; // box sector of each slot
        int n_classes = 1;           // full-operator Gauss-Seidel: sector colour classes
        // K-cycle coarse solve (cycle_type 1): vectors of the next level's size, the dot
        // products and the step coefficients
        DeviceArray<double> kg, kv1, kw1, kv2, kw2, kr, ke, kdots, kcoef, kpartials;
    };
    MultigridOptions opt;
    double shift = 0.0;
    int max_depth = 0;
    bool full_ = false;
    std::vector<std::unique_ptr<Level>> levels;
    DeviceArray<double> lgf;
    std::shared_ptr<Binomials> binom;

    Multigrid(const Space &space, const Model &model, double shift, const MultigridOptions &opt);
    // The full-operator hierarchy of the paper driver (rdme/cpp/rdme_full_multigrid.cpp:348-560,
    // 819-850): every level is the whole box on a grid coarsened d times, with diffusivities
    // doubled per level and the reactions of level_models[d] (the caller tabulates the rates at
    // that level's voxel volume; level_models[0] is the fine model); the coarsest level, where
    // the grid stops coarsening, is solved densely as one block. Weighted Jacobi smoothing, or
    // Gauss-Seidel over (sector colour class x checkerboard colour) passes: reactions couple
    // states of one checkerboard colour, so the sectors they couple get different classes.
    Multigrid(const Space &space, const std::vector<const Model *> &level_models, double shift,
              const MultigridOptions &opt);
    [[nodiscard]] bool full_operator() const { return full_; }

  private:
    Multigrid(const Space &space, const Model &model, double shift, const MultigridOptions &opt,
              const std::vector<const Model *> *level_models);
    // the K-cycle's coarse correction at depth d + 1 (two GCR steps); returns its device vector
    double *kcycle_coarse(int d, cudaStream_t stream);

  public:
    ~Multigrid() override;
    // x = M b (FP64 in and out; FP32 inside when opt.precision == 1)
    void apply(const double *b, double *x, cudaStream_t stream) override;
    [[nodiscard]] bool varies() const override { return opt.precision != 0 || opt.cycle_type == 1; }
    // the same for nb <= opt.batch right-hand sides at once: column c of b at b + c * ldb,
    // of x at x + c * ldx; one cycle serves all columns
    void apply_batch(const double *b, std::int64_t ldb, double *x, std::int64_t ldx, int nb,
                     cudaStream_t stream);
    // the FP32 batched cycle's interleaved lanes: pack nb FP64 columns (c at c * ldx) into y,
    // lanes >= nb zero; unpack lanes < nb into FP64 columns at c * ldy
    static cudaError_t pack_lanes(const double *x, std::int64_t ldx, int nb, float *y,
                                  std::int64_t n, cudaStream_t stream);
    static cudaError_t unpack_lanes(const float *x, std::int64_t n, int nb, double *y,
                                    std::int64_t ldy, cudaStream_t stream);
    // bytes of work vectors one cycle needs, each vector aligned to 256 bytes
    [[nodiscard]] std::size_t scratch_bytes() const;
    // the same cycle with every work vector carved from caller-given device memory of at
    // least scratch_bytes(); plain launches, nothing allocated
    void apply_in(const double *b, double *x, void *scratch, std::size_t bytes,
                  cudaStream_t stream);
    [[nodiscard]] int n_levels() const { return static_cast<int>(levels.size()); }
    [[nodiscard]] int levels_of_sector(int k) const;
    // FP64 hooks on one depth: population_transfer restrict (direction 0) or prolong (1)
    // between depth d and d + 1, and y = (shift I - Q_d) x on depth d
    void transfer(int d, int direction, const double *in, double *out, cudaStream_t stream);
    void apply_system(int d, const double *x, double *y, cudaStream_t stream);
    // one sweep of the level's smoother on (b, x) at depth d, FP64 preconditioners only
    // (the Jacobi update of multigrid.hpp:309-317, or one colour pass pair, or one ILU(0) sweep)
    void smooth(int d, const double *b, double *x, cudaStream_t stream);

  private:
    // carve: six work-vector pointers per level in caller memory (apply_in), else null
    template <typename T>
    T *cycle(int d, cudaStream_t stream, void *const *carve = nullptr);
    template <typename T>
    void ilu_pivots();
    template <typename T>
    void ilu_sweep(Level &L, RowParams<T> p, T *x, const T *rhs, T *work, cudaStream_t stream);
    template <typename T>
    T *buf(Level &L, int which, void *const *carve_level = nullptr);
    template <typename T>
    const T *weights(const Level &L) const;
    void build_aggregates(Level &L, const std::vector<int> &parent, int coarse_voxels);
    template <typename T>
    void aggregate_smooth(Level &L, const T *rhs, T *x, T *scratch, int sweeps, bool reverse,
                          bool from_zero, cudaStream_t stream);
    void build_transfers();
    void ensure_graph(int nb);
    // the captured cycle for each batch width, and its kernel nodes
    std::vector<cudaGraphExec_t> graph_exec_;
    std::vector<std::uint64_t> graph_kernels_;
    int nb_ = 1; // columns the cycle being recorded or run serves
};

struct GmresOptions {
    double tolerance = 1e-8; // absolute, on the Euclidean residual norm
    std::int64_t max_iterations = 1000;
    int restart = 30;
    int flexible = 0; // keep Z_j = M v_j (required for the FP32 preconditioner)
};

struct SolverResult {
    std::int64_t iterations = 0;
    double residual = 0.0;
    int converged = 0;
    int status = kOk;
};

// workspace of restarted (F)GMRES for one system size
struct Krylov {
    std::int64_t n = 0, ld = 0;
    int m = 0;
    bool flexible = false;
    DeviceArray<double> V, Z, w, r, t, partials, small;
    DeviceArray<int> skip; // the selective re-orthogonalisation's decision
    ArnoldiState st;
    double *report_host = nullptr; // pinned, 3 slots of 4
    cudaEvent_t step_done[2] = {nullptr, nullptr};
    Krylov(std::int64_t n, int m, bool flexible);
    ~Krylov();
    Krylov(const Krylov &) = delete;
    Krylov &operator=(const Krylov &) = delete;
};

// the stationary iteration x <- x + M (b - A x) on A = shift I - Q (the paper driver's
// multigrid method, rdme/cpp/rdme_full_multigrid.cpp:1190-1215) until ||b - A x||_2 <= tol;
// iterations = cycles applied
SolverResult stationary(const Generator &A, double shift, Preconditioner &M, const double *b,
                        double *x, double tol, std::int64_t max_cycles, cudaStream_t stream);

// right-preconditioned restarted GMRES (Saad Alg. 9.5) or FGMRES (Alg. 9.6) on
// A = shift I - Q with classical Gram-Schmidt and one re-orthogonalisation
SolverResult gmres(const Generator &A, double shift, Preconditioner *M, const double *b,
                   double *x, const GmresOptions &opt, Krylov &ws, cudaStream_t stream);

// Workspace of FGMRES for nb right-hand sides advanced in lockstep. Basis vector j of column
// c sits at V + (j * nb + c) * ld (and Z likewise), so step j of every column is one strided
// block for the batched operator and multigrid, and column c's basis is strided by nb * ld
// for its Gram-Schmidt passes.
struct KrylovBatch {
    std::int64_t n = 0, ld = 0;
    int m = 0, nb = 0;
    DeviceArray<double> V, Z, w, r, partials, small;
    DeviceArray<double> reports;      // 4 per column: the last batched step's Givens reports
    std::int64_t small_stride = 0;    // doubles between consecutive columns' Arnoldi states
    std::vector<ArnoldiState> st;
    double *report_host = nullptr; // pinned: two slots (steps j and j + 1) of 4 per column
    cudaEvent_t step_done[2] = {nullptr, nullptr};
    KrylovBatch(std::int64_t n, int m, int nb);
    ~KrylovBatch();
    KrylovBatch(const KrylovBatch &) = delete;
    KrylovBatch &operator=(const KrylovBatch &) = delete;
};

// FGMRES on nb <= ws.nb right-hand sides at once (column c of b and x at c * ws.ld): one
// batched operator apply and one batched multigrid cycle per step serve every column, and one
// launch per Gram-Schmidt pass serves every running column (per-column arithmetic unchanged). Column c stops at its own absolute
// tolerance tol[c] (opt.tolerance is unused); the batch stops when every column has.
std::vector<SolverResult> gmres_batch(const Generator &A, double shift, Multigrid &M,
                                      const double *b, double *x, int nb, const double *tol,
                                      const GmresOptions &opt, KrylovBatch &ws,
                                      cudaStream_t stream);

} // namespace mkb
