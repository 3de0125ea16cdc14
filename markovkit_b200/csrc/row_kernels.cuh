// Launch interface of the row kernels: every pass of the generator and of the multigrid
// smoothers is one launch over a tile list that covers a level space.
#pragma once

#include "generator_row.cuh"
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

enum RowMode : int {
    kApplyQ = 0,          // y = Q x
    kApplyShifted,        // y = shift x - Q x
    kResidual,            // y = b - (shift x - Q x)
    kJacobiZero,          // y = omega b / (shift + exit)       (a Jacobi sweep from x = 0)
    kJacobi,              // y = x + omega (b - A x) / (shift + exit)
    kGaussSeidel,         // x_i = (b_i + in_i) / (shift + exit_i) for states of one colour
    kExitLeak,            // y = exit, aux = leak
    kResidualRestrict,    // r = b - A x; coarse[c(i)] += r (or aux = r on terminal sectors)
    kProlongAdd,          // y += weight * coarse[c(i)]
    kDiagonal,            // y = shift + exit
    kRestrict,            // coarse[c(i)] += x_i                (population_transfer::restrict)
    kProlong,             // y_i = weight_i * coarse[c(i)]      (population_transfer::prolong)
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
    const T *x = nullptr;
    const T *b = nullptr;
    T *y = nullptr;
    T *aux = nullptr;
    T *coarse = nullptr;
    const T *piv = nullptr; // ILU(0) pivots of the second colour
    T shift = 0;
    T omega = 0;
    int colour = 0;
    int n_tiles = 0;
    int mode = kApplyShifted;
    // right-hand sides served at once (1..kRowBatch): column c of x, b, y and aux starts at
    // c * ldv, column c of coarse at c * ldc
    int nb = 1;
    std::int64_t ldv = 0;
    std::int64_t ldc = 0;
};

constexpr int kRowBatch = 4; // widest batch of the instantiated kernels

// the largest species total the kernels handle: 64 with one species, 16 with more
int mol_cap_for(int n_species, int max_species_total);

// one pass over every tile; (S, cap) select the kernel's state shape
template <typename T>
cudaError_t launch_rows(RowMode mode, int S, int cap, const RowParams<T> &p, cudaStream_t stream);
cudaError_t launch_rows_f64(const RowParams<double> &p, int S, int cap, cudaStream_t stream);
cudaError_t launch_rows_f32(const RowParams<float> &p, int S, int cap, cudaStream_t stream);
// the batched instantiations (p.nb > 1)
cudaError_t launch_rows_f64_batch(const RowParams<double> &p, int S, int cap, cudaStream_t stream);
cudaError_t launch_rows_f32_batch(const RowParams<float> &p, int S, int cap, cudaStream_t stream);

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
