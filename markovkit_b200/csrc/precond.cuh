// Fixed right preconditioners of gmres() beside the multigrid, the ones the reference's RDME
// benchmark compares it with (examples/rdme_multigrid_benchmark.cpp:109-115):
//   num::jacobi_preconditioner(inverse_diagonal)  z = d .* v
//   num::ilu0_preconditioner(A)                   z = U^-1 L^-1 v, ILU(0) of A in its natural
//                                                 row order
// and a host callback standing in for any other operator with apply(x, y).
//
// ILU(0) on the device. The factorisation is the row-wise IKJ form (Saad, Iterative Methods for
// Sparse Linear Systems, 2nd ed., Alg. 10.4): for each k < i in row i's pattern, ascending,
// l_ik = a_ik / u_kk, then a_ij -= l_ik u_kj for the j > k in both rows' patterns. Row i reads
// only rows k < i that it references, so rows fall into levels (level(i) = 1 + the largest
// level of the rows it references, 0 with none), and every row of a level is factored at once
// by one thread once the earlier levels are final. The forward solve L y = v uses the same
// levels; the backward solve U z = y uses the mirrored ones. Runs of consecutive levels of at
// most kNarrowRows rows go to one CUDA block that steps through them between block barriers,
// so a deep, thin schedule costs one launch per run instead of one per level; a level wider
// than that, or with more entries than kNarrowWork, gets its own grid, and in the triangular
// solves a warp per row when its rows are long (the one-molecule rows of a box hold an entry
// per voxel). Every update is a fused multiply-add (fma(-l, u, a)).
#pragma once

#include "engine.hpp"

#include <cstdint>
#include <vector>

namespace mkb {

// z = d .* v, d the inverse diagonal given at construction
struct DiagonalPreconditioner final : Preconditioner {
    DeviceArray<double> d;
    DiagonalPreconditioner(const double *inverse_diagonal_host, std::int64_t n);
    void apply(const double *v, double *z, cudaStream_t stream) override;
};

// rows of one triangular sweep grouped by level; a segment is a run of levels launched together
struct LevelSchedule {
    struct Segment {
        std::int64_t l0 = 0, l1 = 0; // levels [l0, l1)
        std::int64_t rows = 0;
        bool wide = false;           // one level over a grid, else one block steps the levels
        bool warp = false;           // wide, with rows long enough for a warp each (solves)
    };
    DeviceArray<int> order;                // rows by level
    DeviceArray<std::int64_t> level_ptr;   // level l: order[level_ptr[l] .. level_ptr[l + 1])
    std::vector<std::int64_t> h_level_ptr;
    std::vector<Segment> segments;
    [[nodiscard]] std::int64_t levels() const {
        return h_level_ptr.empty() ? 0 : static_cast<std::int64_t>(h_level_ptr.size()) - 1;
    }
};

struct Ilu0Preconditioner final : Preconditioner {
    static constexpr int kNarrowRows = 4096;     // levels at most this wide share one block,
    static constexpr int kNarrowWork = 1 << 16;  // if their entries are at most this many
    static constexpr int kWarpRowLength = 32;    // a wide level whose longest row is longer
                                                 // than this runs a warp per row
    // the factors in A's pattern (each row's columns ascending): L strictly below the diagonal
    // (unit diagonal implied), U on and above it
    DeviceArray<std::int64_t> ptr, diag;
    DeviceArray<int> col;
    DeviceArray<double> val;
    LevelSchedule lower, upper;
    DeviceArray<double> y; // L^-1 v
    // A in CSR on the host: row_ptr[n + 1], col/val[row_ptr[n]]; each row's columns strictly
    // ascending and its diagonal present (MK_EINVAL otherwise); MK_ESINGULAR on a zero or
    // non-finite pivot
    Ilu0Preconditioner(std::int64_t n, const std::int64_t *row_ptr, const std::int64_t *col,
                       const double *val, cudaStream_t stream);
    void apply(const double *v, double *z, cudaStream_t stream) override;
};

// z = fn(ctx, v) on the host: v is copied out, fn runs on the calling thread, z copied back.
// fn returns 0 on success; anything else fails the solve with MK_EINVAL.
struct HostPreconditioner final : Preconditioner {
    using Fn = int (*)(void *ctx, const double *v, double *z, std::int64_t n);
    Fn fn = nullptr;
    void *ctx = nullptr;
    double *hv = nullptr, *hz = nullptr; // pinned
    HostPreconditioner(std::int64_t n, Fn fn, void *ctx);
    ~HostPreconditioner() override;
    void apply(const double *v, double *z, cudaStream_t stream) override;
};

} // namespace mkb
