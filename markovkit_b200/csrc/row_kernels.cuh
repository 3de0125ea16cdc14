// Launch interface of the row kernels: every pass of the generator and of the multigrid
// smoothers is one launch over a tile list that covers a level space.
#pragma once

#include "generator_row.cuh"
#include "stencil_tables.hpp"
#include <cuda_runtime.h>

namespace mkb {

// A tile is a block's work: `count` consecutive states of one sector, one per thread
// (kind 0), or one per warp for rows with all-voxel in-jumps (kind 1).
struct Tile {
    std::int64_t local0 = 0;
    int sector = 0;
    int kind = 0;
    int count = 0;
    int pad = 0;
};
constexpr int kRowBlock = 256;
constexpr int kWarpRows = kRowBlock / 32;
constexpr int kHeavyGroupRows = 8; // rows of a kind-4 (grouped heavy) tile

constexpr int kRowBatch = 4; // widest batch of the instantiated kernels

enum RowMode : int {
    kApplyQ = 0,          // y = Q x
    kApplyShifted,        // y = shift x - Q x
    kResidual,            // y = b - (shift x - Q x)
    kJacobiZero,          // y = omega b / (shift + exit)       (a Jacobi sweep from x = 0)
    kJacobi,              // y = x + omega (b - A x) / (shift + exit)
    kGaussSeidel,         // x_i = (b_i + in_i) / (shift + exit_i) for states of one colour
    kExitLeak,            // y = exit, aux = leak
    kDiagonal,            // y = shift + exit
    kCoarseIndex,         // idx_i = coarse state of fine state i (-1 on terminal sectors) and
                          // wout_i = its prolongation weight (multigrid set-up)
    // red-black ILU(0) of A = shift I - Q on a bipartite (diffusion-only) level, colour 0 first:
    // with A = [D0 A01; A10 D1], L = [I 0; A10 D0^-1 I], U = [D0 A01; 0 P1], and the pivots
    // P1 = D1 - diag(A10 D0^-1 A01). One sweep x += U^-1 L^-1 (b - A x) is three passes:
    kIluPivot,            // colour 1: y = shift + exit - sum_j rate(j->i) rate(i->j) / aux_j (aux = diagonal)
    kIluFirst,            // colour 0: aux = (b - A x) / (shift + exit)
    kIluSecond,           // colour 1: z = (b - A x + sum_j rate(j->i) aux_j) / piv; aux = z; y = x + z
    kIluThird,            // colour 0: y = x + aux + sum_j rate(j->i) aux_j / (shift + exit)
    kRowModeCount
};

template <typename T>
struct RowParams {
    BinomTable B;
    const SectorDesc *sectors = nullptr;
    const Tile *tiles = nullptr;
    ModelView<T> md;
    TransferView tv;
    StencilView<T> sv;
    const T *x = nullptr;
    const T *b = nullptr;
    T *y = nullptr;
    T *aux = nullptr;
    const T *piv = nullptr; // ILU(0) pivots of the second colour
    int *idx = nullptr;     // kCoarseIndex output
    double *wout = nullptr; // kCoarseIndex output
    T shift = 0;
    T omega = 0;
    int colour = 0;
    int n_tiles = 0;
    int mode = kApplyShifted;
    // right-hand sides served at once (1..kRowBatch): column c of x, b, y and aux starts at
    // c * ldv (the interleaved FP32 batch keeps entry (i, c) at i * kRowBatch + c)
    int nb = 1;
    std::int64_t ldv = 0;
    // batched requests of one problem with different shifts: column c uses col_shift[c], and
    // with piv_per_col its ILU(0) pivots sit at column c of piv (laid out like x)
    // Gauss-Seidel of the full operator: only sectors of this colour class (-1: all)
    int sector_class = -1;
    int per_col_shift = 0;
    int piv_per_col = 0;
    T col_shift[kRowBatch] = {};
};

// the largest species total the kernels handle: 64 with one species, 16 with more
int mol_cap_for(int n_species, int max_species_total);

// one pass over every tile; (S, cap) select the kernel's state shape
template <typename T>
cudaError_t launch_rows(RowMode mode, int S, int cap, const RowParams<T> &p, cudaStream_t stream);
// the general row kernel for every shape (p.nb > 1 selects the batched instantiations)
cudaError_t launch_rows_f64(const RowParams<double> &p, int S, int cap, cudaStream_t stream);
cudaError_t launch_rows_f32(const RowParams<float> &p, int S, int cap, cudaStream_t stream);

// The stencil row kernel (stencil_row.cuh): light rows of structured-grid levels whose state
// shape is one species of at most four molecules or two species of at most one, for the passes
// of the solve (kApplyQ .. kGaussSeidel and the ILU sweeps). p.tiles lists only such rows.
bool stencil_shape(int S, int cap);
bool stencil_mode(int mode);
cudaError_t launch_stencil_rows_f64(const RowParams<double> &p, int S, int cap, cudaStream_t stream);
cudaError_t launch_stencil_rows_f32(const RowParams<float> &p, int S, int cap, cudaStream_t stream);
// Rows of one species of cap <= 2 whose in-jumps come from every voxel, in the operator passes
// (kApplyQ, kApplyShifted, kResidual): a warp or a block per row with closed-form source ranks.
bool pair_heavy_mode(int mode);
cudaError_t launch_pair_heavy_rows_f64(const RowParams<double> &p, cudaStream_t stream);
cudaError_t launch_pair_heavy_rows_f32(const RowParams<float> &p, cudaStream_t stream);

// Rows of two-molecule sectors of one species (every pair u0 <= u1 of V voxels), a block per
// pair of triangle rows (kind-3 tiles, local0 = the pair index), for the stencil passes; the
// results equal the stencil kernel's bit for bit.
cudaError_t launch_pair_strip_rows_f64(const RowParams<double> &p, cudaStream_t stream);
cudaError_t launch_pair_strip_rows_f32(const RowParams<float> &p, cudaStream_t stream);
// Rows of one molecule whose heavy in-jumps come from the pair sector, eight rows a block
// (kind-4 tiles), in the operator passes: the sources of the group's rows for one voxel w sit
// side by side, so the reads of the pair sector coalesce.
cudaError_t launch_pair_heavy_group_rows_f64(const RowParams<double> &p, cudaStream_t stream);
cudaError_t launch_pair_heavy_group_rows_f32(const RowParams<float> &p, cudaStream_t stream);

namespace detail {
// the general row kernel of one state shape (row_kernels_impl.cuh, instantiated per shape by
// row_kernels_inst.cu)
template <typename T, int NS, int TMAX, int NB>
cudaError_t launch_shape(const RowParams<T> &p, cudaStream_t stream);
// the stencil row kernel of the shape (S, cap) (stencil_rows.cu, one unit per T and NB)
template <typename T, int NB>
cudaError_t launch_stencil(const RowParams<T> &p, int S, int cap, cudaStream_t stream);
// the pair-form kernel for rows with in-jumps from every voxel (one species of cap <= 2)
template <typename T, int NB>
cudaError_t launch_pair_heavy(const RowParams<T> &p, cudaStream_t stream);
// the pair-strip kernel for the rows of two-molecule sectors of one species
template <typename T, int NB>
cudaError_t launch_pair_strip(const RowParams<T> &p, cudaStream_t stream);
// the grouped heavy-row kernel for rows of one molecule
template <typename T, int NB>
cudaError_t launch_pair_heavy_group(const RowParams<T> &p, cudaStream_t stream);
} // namespace detail

struct TerminalBlock {
    std::int64_t begin = 0;      // first row in the level space
    std::int64_t inv_offset = 0; // offset of the n x n inverse
    int n = 0;
    int pad = 0;
};

// x[begin + p] += sum_q inv[p][q] r[begin + q] for every terminal block (max_n: the largest);
// entry q of r and x at q * stride
template <typename T>
cudaError_t launch_terminal(const TerminalBlock *blocks, int n_blocks, int max_n, const T *inv,
                            const T *r, T *x, int stride, cudaStream_t stream);

// bit-exact state indexing on the device
cudaError_t launch_unrank(const BinomTable &B, const SectorDesc *sectors, int n_sectors, int S,
                          int V, const std::int64_t *index, std::int64_t count, int *states,
                          cudaStream_t stream);
cudaError_t launch_rank(const BinomTable &B, const SectorDesc *sectors, int n_sectors,
                        const int *max_totals, int is_box, int S, int V, const int *states,
                        std::int64_t count, std::int64_t *index, cudaStream_t stream);

} // namespace mkb
