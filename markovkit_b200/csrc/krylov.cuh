// Krylov building blocks on sm_100a: fused classical Gram-Schmidt passes, norms, vector
// updates and the small Hessenberg / Givens state of (F)GMRES. Reductions are two-stage with
// a fixed grid and fixed summation order, so results are bitwise reproducible run to run.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mkb {

constexpr int kDotBlocks = 148 * 4; // one wave of 4 blocks per SM
constexpr int kDotThreads = 256;
constexpr int kMaxFusedBasis = 32;  // basis vectors handled by the fused CGS kernels

// partials[k * kDotBlocks + block] for k < K, then out[k] = sum over blocks (fixed order)
//   mode 0: out[k] = <V_k, w>
//   mode 1: w -= sum_k coef[k] V_k, then out[k] = <V_k, w_new>
//   mode 2: w -= sum_k coef[k] V_k, then out[0] = <w_new, w_new>
//   mode 3: w -= sum_k coef[k] V_k only
// K <= kMaxFusedBasis; longer bases are processed in chunks by the caller.
// One Gram-Schmidt step with selective re-orthogonalisation (Daniel, Gragg, Kaufman, Stewart,
// Math. Comp. 30, 1976): h1 = V^T w, w -= V h1; a second pass h2 = V^T w, w -= V h2 only when
// ||w|| dropped below 1/sqrt(2) of its value, decided on the device (h2 = 0 and the second
// pass's kernels return at once otherwise); hn = <w, w> after the step. K < kMaxFusedBasis
// (h1 and h2 hold K + 1 entries: entry K is a norm); skip is one device int of scratch.
cudaError_t cgs_dgks(const double *V, std::int64_t ld, int K, double *w, std::int64_t n,
                     double *partials, double *h1, double *h2, double *hn, int *skip,
                     cudaStream_t stream);

cudaError_t cgs_pass(int mode, const double *V, std::int64_t ld, int K, double *w, std::int64_t n,
                     const double *coef, double *partials, double *out, cudaStream_t stream);

// out[0] = <a, b>
cudaError_t dot(const double *a, const double *b, std::int64_t n, double *partials, double *out,
                cudaStream_t stream);

// y = x * (*scale)           (scale read on the device)
cudaError_t scale_copy(const double *x, const double *scale, double *y, std::int64_t n,
                       cudaStream_t stream);
// y += sum_k coef[k] V_k     (coef read on the device)
cudaError_t multi_axpy(const double *V, std::int64_t ld, int K, const double *coef, double *y,
                       std::int64_t n, cudaStream_t stream);
// y = sum_k coef[k] V_k
cudaError_t multi_combine(const double *V, std::int64_t ld, int K, const double *coef, double *y,
                          std::int64_t n, cudaStream_t stream);
// y = a x + y with a host scalar
cudaError_t axpy(double a, const double *x, double *y, std::int64_t n, cudaStream_t stream);
template <typename A, typename B>
cudaError_t convert(const A *x, B *y, std::int64_t n, cudaStream_t stream);

// Hessenberg / Givens state of one restart cycle, in device memory
struct ArnoldiState {
    double *H = nullptr;      // (m + 1) x m, column-major: H[j * (m + 1) + i]
    double *cs = nullptr;     // m
    double *sn = nullptr;     // m
    double *g = nullptr;      // m + 1
    double *y = nullptr;      // m
    double *h1 = nullptr;     // m + 1: first Gram-Schmidt coefficients
    double *h2 = nullptr;     // m + 1: second (re-orthogonalisation) coefficients
    double *hn = nullptr;     // 1: <w, w> after the second pass
    double *inv_hn = nullptr; // 1
    double *beta = nullptr;   // 1: <r, r> on entry, then 1 / ||r||
    double *report = nullptr; // 4: |g_{j+1}|, ||w||, breakdown flag, spare
    int m = 0;
};

// The running columns of a lockstep batch (batched FGMRES): column c's basis vector k sits at
// V + c * col + k * vstride, its w at w + c * col, its Arnoldi state at st's pointers + c * small
// (offsets in doubles); partials hold nb * kDotBlocks * kMaxFusedBasis doubles; bit c of mask
// selects column c.
struct ColumnBatch {
    double *V = nullptr;
    std::int64_t vstride = 0;
    double *w = nullptr;
    std::int64_t col = 0;
    ArnoldiState st;
    std::int64_t small = 0;
    double *partials = nullptr;
    double *reports = nullptr; // 4 per column, contiguous: the step's Givens report
    int nb = 0;
    unsigned mask = 0;
    std::int64_t n = 0;
};

// Step j's classical Gram-Schmidt with one re-orthogonalisation for every selected column at
// once (K = j + 1 <= kMaxFusedBasis): h1 = V^T w; w -= V h1, h2 = V^T w; w -= V h2,
// hn = <w, w>; the Givens column j (as arnoldi_column, its report also copied to reports);
// and, when next, V_{j+1} = w / sqrt(hn). One launch per pass serves every column; per column
// the arithmetic is that of cgs_pass, arnoldi_column and scale_copy, so the results are the
// same bit for bit.
cudaError_t cgs_step_batch(const ColumnBatch &b, int j, bool next, cudaStream_t stream);

// g = (||r||, 0, ...), beta <- 1/||r|| (reads beta = <r, r>)
cudaError_t arnoldi_start(const ArnoldiState &s, cudaStream_t stream);
// fold column j (h1 + h2, sqrt(hn)) into H, rotate, update g; report |g_{j+1}|
cudaError_t arnoldi_column(const ArnoldiState &s, int j, cudaStream_t stream);
// y = H_k^{-1} g_k (upper triangular, k columns)
cudaError_t arnoldi_solve(const ArnoldiState &s, int k, cudaStream_t stream);

} // namespace mkb
