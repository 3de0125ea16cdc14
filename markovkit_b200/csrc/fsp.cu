// Batched Krylov FSP (markovkit/fsp.hpp:190-254) in one persistent sm_100a kernel.
//
// Each block takes instances from an atomic queue (the host orders them largest first) and runs
// the reference's whole attempt loop on one instance with no host round trip:
//   expand the support by `layers` rings inside the box region (fsp.hpp:44-59);
//   w = expv(tau, Q, p) with Q the absorbing generator of the support (generator.hpp:27-44):
//       every positive jump to a non-negative state counts in the exit rate, and only jumps
//       between supported states are off-diagonal entries;
//   halve tau while sum(max(0, w)) < 1 - tol (t + tau) / T and tau > 1e-14 (fsp.hpp:224-231);
//   otherwise dp = Q w, p = max(0, w), drop states with p < drop_probability and
//   |dp| < drop_derivative, renormalise, t += tau, tau = min(tau * growth, T - t).
// expv is Sidje's Expokit controller as the numerics library is called (fsp.hpp:223): Krylov
// dimension m, the augmented (m+2)-square Hessenberg, a Pade (6,6) exponential with scaling and
// squaring, the two-term error estimate, safety factors 0.9 and 1.2, break-down below 1e-7.
//
// Data layout. The support is a compact list of slots with a box-to-slot map, in the
// reference's order: an expansion ring appends new states in the order the reference discovers
// them (support slot, then reaction; the first discoverer of a state wins, found with an atomic
// minimum over candidate numbers), and dropped states are compacted out in order. After the
// expansion, each attempt assembles Q on its support as R neighbour slots and coefficients per
// state plus the exit rate (reaction-major arrays), as the reference assembles its generator,
// so an apply is one gather per reaction. The assembled operator, the Krylov work vectors and
// the basis go to the block's shared-memory arena in that order of priority, each wherever it
// fits for the attempt's support size, else to the block's global workspace.
//
// One Arnoldi step is three block-wide phases with one barrier each: (1) the apply, which also
// writes the basis vector V_j = p / ||p|| of the previous step and accumulates the first
// Gram-Schmidt projections <V_i, Q V_j>; (2) the first subtraction fused with the second
// projections; (3) the second subtraction fused with the norm. Reductions leave per-warp
// partials in one of two alternating buffers, so each needs a single barrier.
//
// The Pade (6,6) approximant r(X) = q(X)^-1 p(X) of the scaled Hessenberg is formed from X^2,
// X^4, X^6 and one product for the odd part, and q(X) F = p(X) is solved by Gauss-Jordan
// elimination spread over the whole block, one barrier per pivot: ||I - q(X)|| <= 0.28 when
// ||X|| <= 1/2, so q(X) is strictly diagonally dominant and needs no row exchanges.
// Every loop is bounded; no thread waits on another block.
#include "fsp.cuh"
#include "launch_count.hpp"

#include <cmath>

namespace mkb {

namespace {

constexpr int kMaxWarps = 16;
constexpr int kBasis = kFspMaxKrylov + 1;
constexpr int kE = 32;               // side of the small dense matrices in shared memory
constexpr int kNoOwner = 0x7fffffff;
constexpr int kSubstepLimit = 100000;
constexpr std::int64_t kAttemptLimit = 1000000;

static_assert(sizeof(FspInstance) % 4 == 0, "instance is copied as words");

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

struct Shared {
    FspInstance in;
    double H[kE * kE];
    double M[7][kE * kE];            // the small exponential's matrices
    double red[2][kMaxWarps * kE];   // alternating per-warp partials
    double hw[kMaxWarps][kE];        // each warp's copy of the latest projections
    double h1[kE];                   // first projections, kept for the Hessenberg column
    int i[8];
    int scan[kMaxWarps + 1];
    int hist[256];            // radix-select histogram of the adaptive pruning
    unsigned long long key;   // the select's prefix, broadcast
    int clipped;              // species whose bound an expansion met (bit mask)
};

struct Ctx {
    const FspInstance *in; // the block's shared copy
    const double *rate;
    // the block's global workspace
    double *gV, *prob, *gw, *gbuf0, *gbuf1, *gtmp, *gdiag, *gcoef;
    int *b2s, *s2b, *itmp, *owner, *gnbr;
    std::int64_t cap;
    // this attempt's placement (shared arena or global workspace)
    double *V, *w, *buf0, *buf1, *tmp, *diag, *coef;
    int *nbr;
    std::int64_t vs, es; // strides of basis vectors and of operator arrays
    unsigned char *arena;
    std::size_t arena_bytes;
    int parity; // which partials buffer the next reduction uses
};

// the block's sum (or max) of v on every thread; one barrier
template <int NT, bool MAX>
__device__ double block_reduce(Shared &sh, Ctx &c, double v) {
    constexpr int W = NT / 32;
    v = MAX ? warp_max(v) : warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *red = sh.red[c.parity];
    c.parity ^= 1;
    if (lane == 0) {
        red[warp] = v;
    }
    __syncthreads();
    double t = red[0];
#pragma unroll
    for (int w = 1; w < W; ++w) {
        t = MAX ? fmax(t, red[w]) : t + red[w];
    }
    return t;
}

// Reduces acc[q] over the warp (q < 16) with 16 shuffles: afterwards lane l holds the warp
// total of one value, numbered by its lane bits 4..1. Writes the totals of values
// k0 + q < K to red[warp * kE + k0 + q].
__device__ __forceinline__ void stash_partials(double *red, double (&acc)[16], int k0, int K) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const bool hi = lane & 16;
        const double send = hi ? acc[q] : acc[q + 8];
        const double keep = hi ? acc[q + 8] : acc[q];
        acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool hi = lane & 8;
        const double send = hi ? acc[q] : acc[q + 4];
        const double keep = hi ? acc[q + 4] : acc[q];
        acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const bool hi = lane & 4;
        const double send = hi ? acc[q] : acc[q + 2];
        const double keep = hi ? acc[q + 2] : acc[q];
        acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {
        const bool hi = lane & 2;
        const double send = hi ? acc[0] : acc[1];
        const double keep = hi ? acc[1] : acc[0];
        acc[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], 1);
    const int q = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 +
                  ((lane >> 1) & 1);
    if ((lane & 1) == 0 && k0 + q < K) {
        red[warp * kE + k0 + q] = acc[0];
    }
}

// after the partials of K values are stashed: one barrier, then every warp sums them into its
// own row sh.hw[warp] (lane i holds value i), visible to the warp on return
template <int NT>
__device__ void finish_projections(Shared &sh, const double *red, int K) {
    constexpr int W = NT / 32;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane < K) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            t += red[w * kE + lane];
        }
        sh.hw[warp][lane] = t;
    }
    __syncwarp();
}

__device__ __forceinline__ void zero16(double (&acc)[16]) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        acc[q] = 0.0;
    }
}

// Order-preserving compaction of [0, L): emit(i, dest) for every i with pred(i), dest counting
// the kept ones before i. Returns the number kept (all threads).
template <int NT, typename Pred, typename Emit>
__device__ int compact(Shared &sh, int L, Pred pred, Emit emit) {
    constexpr int W = NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int base = 0;
    for (int c0 = 0; c0 < L; c0 += NT) {
        const int i = c0 + static_cast<int>(threadIdx.x);
        const int f = (i < L && pred(i)) ? 1 : 0;
        int incl = f;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, off);
            incl += lane >= off ? y : 0;
        }
        if (lane == 31) {
            sh.scan[warp] = incl;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int w = 0; w < W; ++w) {
                const int t = sh.scan[w];
                sh.scan[w] = acc;
                acc += t;
            }
            sh.scan[W] = acc;
        }
        __syncthreads();
        if (f) {
            emit(i, base + sh.scan[warp] + incl - 1);
        }
        base += sh.scan[W];
        __syncthreads();
    }
    return base;
}

__device__ __forceinline__ void coords(const FspInstance &in, int i, int (&x)[kFspMaxSpecies]) {
#pragma unroll
    for (int s = 0; s < kFspMaxSpecies; ++s) {
        x[s] = s < in.S ? (i / in.stride[s]) % (in.bound[s] + 1) : 0;
    }
}

// ---- placement and assembly -------------------------------------------------------------

__device__ __forceinline__ void *take(Ctx &c, std::size_t &off, std::size_t bytes) {
    bytes = (bytes + 15) & ~std::size_t(15);
    if (off + bytes > c.arena_bytes) {
        return nullptr;
    }
    void *p = c.arena + off;
    off += bytes;
    return p;
}

// where this attempt's operator, vectors and basis live (same answer on every thread)
__device__ void place(Ctx &c, int n, int m) {
    const int R = c.in->R;
    std::size_t off = 0;
    const std::size_t nd = static_cast<std::size_t>(n) * sizeof(double);
    {
        const std::size_t mark = off;
        auto *coef = static_cast<double *>(take(c, off, nd * R));
        auto *diag = static_cast<double *>(take(c, off, nd));
        auto *nbr = static_cast<int *>(take(c, off, static_cast<std::size_t>(n) * R * sizeof(int)));
        if (diag && (R == 0 || (coef && nbr))) {
            c.coef = coef;
            c.diag = diag;
            c.nbr = nbr;
            c.es = n;
        } else {
            // the global copies are packed at the support's size too (few pages to touch)
            off = mark;
            c.coef = c.gcoef;
            c.diag = c.gdiag;
            c.nbr = c.gnbr;
            c.es = (n + 3) & ~3;
        }
    }
    {
        const std::size_t mark = off;
        auto *w = static_cast<double *>(take(c, off, nd));
        auto *b0 = static_cast<double *>(take(c, off, nd));
        auto *b1 = static_cast<double *>(take(c, off, nd));
        auto *tmp = static_cast<double *>(take(c, off, nd));
        if (w && b0 && b1 && tmp) {
            c.w = w;
            c.buf0 = b0;
            c.buf1 = b1;
            c.tmp = tmp;
        } else {
            off = mark;
            c.w = c.gw;
            c.buf0 = c.gbuf0;
            c.buf1 = c.gbuf1;
            c.tmp = c.gtmp;
        }
    }
    auto *V = static_cast<double *>(take(c, off, nd * (m + 1)));
    if (V) {
        c.V = V;
        c.vs = n;
    } else {
        c.V = c.gV;
        c.vs = (n + 3) & ~3;
    }
}

// Q on the support (generator.hpp:27-44, absorbing): for slot k and reaction r the source
// slot and rate of the jump into k (coefficient 0 and the slot itself when there is none),
// and the exit rate of k over every valid positive jump
// With `reflecting` (the adaptive FSP's generator, boundary::reflecting), the exit rate counts
// only the jumps that land in the support.
template <int NT>
__device__ void assemble(const Ctx &c, int n, bool reflecting = false) {
    const FspInstance &in = *c.in;
    for (int k = threadIdx.x; k < n; k += NT) {
        const int i = c.s2b[k];
        int xi[kFspMaxSpecies];
        coords(in, i, xi);
        double ex = 0.0;
        for (int r = 0; r < in.R; ++r) {
            bool valid = true, inside = true, lands = true;
            int j = i, to = i;
#pragma unroll
            for (int s = 0; s < kFspMaxSpecies; ++s) {
                if (s < in.S) {
                    const int ch = in.change[r][s];
                    valid = valid && xi[s] + ch >= 0;
                    lands = lands && xi[s] + ch <= in.bound[s];
                    const int xs = xi[s] - ch;
                    inside = inside && xs >= 0 && xs <= in.bound[s];
                    j -= ch * in.stride[s];
                    to += ch * in.stride[s];
                }
            }
            const double a = c.rate[static_cast<std::int64_t>(r) * in.box + i];
            if (a > 0.0 && valid && (!reflecting || (lands && c.b2s[to] >= 0))) {
                ex += a;
            }
            int sl = k;
            double coef = 0.0;
            if (inside) {
                const int src = c.b2s[j];
                const double aj = c.rate[static_cast<std::int64_t>(r) * in.box + j];
                if (src >= 0 && aj > 0.0) {
                    sl = src;
                    coef = aj;
                }
            }
            c.nbr[r * c.es + k] = sl;
            c.coef[r * c.es + k] = coef;
        }
        c.diag[k] = ex;
    }
    __syncthreads();
}

// (Q x)_k from the assembled operator
__device__ __forceinline__ double row(const Ctx &c, int R, int k, const double *x) {
    double acc = 0.0;
    for (int r = 0; r < R; ++r) {
        acc += c.coef[r * c.es + k] * x[c.nbr[r * c.es + k]];
    }
    return acc - c.diag[k] * x[k];
}

// ---- Arnoldi phases -------------------------------------------------------------------

// phase 1: V_j = src / div, out = Q V_j, projections <V_i, out> for i <= j into sh.hw
template <int NT>
__device__ void arnoldi_apply(Shared &sh, Ctx &c, int n, const double *src, double div, int j,
                              double *out) {
    const int K = j + 1, R = c.in->R;
    double *Vj = c.V + j * c.vs;
    double *red = sh.red[c.parity];
    c.parity ^= 1;
    double acc[16];
    zero16(acc);
    for (int k = threadIdx.x; k < n; k += NT) {
        const double y = row(c, R, k, src) / div;
        const double vk = src[k] / div;
        Vj[k] = vk;
        out[k] = y;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            if (q < K) {
                acc[q] += (q == j ? vk : c.V[q * c.vs + k]) * y;
            }
        }
    }
    stash_partials(red, acc, 0, K);
    if (K > 16) {
        zero16(acc);
        for (int k = threadIdx.x; k < n; k += NT) {
            const double y = out[k];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                if (16 + q < K) {
                    acc[q] += (16 + q == j ? Vj[k] : c.V[(16 + q) * c.vs + k]) * y;
                }
            }
        }
        stash_partials(red, acc, 16, K);
    }
    finish_projections<NT>(sh, red, K);
}

// phase 2: out -= sum_i h1[i] V_i, then the second projections <V_i, out> into sh.hw
template <int NT>
__device__ void arnoldi_reorthogonalise(Shared &sh, Ctx &c, int n, int K, double *out) {
    const int warp = threadIdx.x >> 5;
    const double *h = sh.hw[warp];
    double *red = sh.red[c.parity];
    c.parity ^= 1;
    double acc[16];
    zero16(acc);
    for (int k = threadIdx.x; k < n; k += NT) {
        // the first 16 basis entries are loaded once for the subtraction and the projection
        double vq[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            vq[q] = q < K ? c.V[q * c.vs + k] : 0.0;
        }
        double v = out[k];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (q < K) {
                v -= h[q] * vq[q];
            }
        }
        for (int i = 8; i < K; ++i) {
            v -= h[i] * c.V[i * c.vs + k];
        }
        out[k] = v;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            if (q < K) {
                acc[q] += (q < 8 ? vq[q] : c.V[q * c.vs + k]) * v;
            }
        }
    }
    // keep the first projections for the Hessenberg column before sh.hw is overwritten
    if (warp == 0 && static_cast<int>(threadIdx.x) < K) {
        sh.h1[threadIdx.x] = h[threadIdx.x];
    }
    stash_partials(red, acc, 0, K);
    if (K > 16) {
        zero16(acc);
        for (int k = threadIdx.x; k < n; k += NT) {
            const double v = out[k];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                if (16 + q < K) {
                    acc[q] += c.V[(16 + q) * c.vs + k] * v;
                }
            }
        }
        stash_partials(red, acc, 16, K);
    }
    finish_projections<NT>(sh, red, K);
}

// phase 3: out -= sum_i h2[i] V_i; returns ||out||^2
template <int NT>
__device__ double arnoldi_finish(Shared &sh, Ctx &c, int n, int K, double *out) {
    const double *h = sh.hw[threadIdx.x >> 5];
    double sq = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        double v = out[k];
        for (int i = 0; i < K; ++i) {
            v -= h[i] * c.V[i * c.vs + k];
        }
        out[k] = v;
        sq += v * v;
    }
    return block_reduce<NT, false>(sh, c, sq);
}

// ---- the small exponential ------------------------------------------------------------

// C = A B for n x n matrices in shared memory (row-major, side kE): each thread computes the
// outputs (i, j) and (i, j + 16) of one row, sharing the loads of A's row
template <int NT>
__device__ void matmul(const double *A, const double *B, double *C, int n) {
    const int j0 = threadIdx.x & 15, j1 = j0 + 16;
    for (int i = threadIdx.x >> 4; i < n; i += NT / 16) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
        for (int k = 0; k < n; ++k) {
            const double a = A[i * kE + k];
            s0 += a * B[k * kE + j0];
            s1 += a * B[k * kE + j1];
        }
        if (j0 < n) {
            C[i * kE + j0] = s0;
        }
        if (j1 < n) {
            C[i * kE + j1] = s1;
        }
    }
    __syncthreads();
}

// F = Q^{-1} P by Gauss-Jordan elimination on [Q | P] (n rows, P in columns 32..), one
// barrier per pivot: every element of step k is computed from step k-1's buffer into the
// other. No row exchanges: Q = I - E with ||E|| <= 0.28 is strictly diagonally dominant by
// rows, so the diagonal is the largest entry of its column at every step and partial pivoting
// would choose it. Q and P are n x n with side kE; A and B hold 32 x 64 each; F gets the result.
template <int NT>
__device__ void gauss_jordan(const double *Q, const double *P, double *A, double *B, double *F,
                             int n) {
    constexpr int S = 2 * kE;
    for (int e = threadIdx.x; e < n * kE; e += NT) {
        const int i = e / kE, j = e - i * kE;
        A[i * S + j] = j < n ? Q[i * kE + j] : 0.0;
        A[i * S + kE + j] = j < n ? P[i * kE + j] : 0.0;
    }
    __syncthreads();
    double *cur = A, *nxt = B;
    for (int k = 0; k < n; ++k) {
        const double rp = 1.0 / cur[k * S + k];
        for (int e = threadIdx.x; e < n * S; e += NT) {
            const int i = e / S, j = e - i * S;
            double v = cur[i * S + j];
            if (i != k) {
                v -= (cur[i * S + k] * rp) * cur[k * S + j];
            }
            nxt[i * S + j] = v;
        }
        __syncthreads();
        double *t = cur;
        cur = nxt;
        nxt = t;
    }
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e / n, j = e - i * n;
        F[i * kE + j] = cur[i * S + kE + j] / cur[i * S + i];
    }
    __syncthreads();
}

// exp(X) for the n x n matrix in sh.M[0] (overwritten); returns the matrix holding the result
template <int NT>
__device__ const double *small_expm(Shared &sh, Ctx &c, int n) {
    double *X = sh.M[0];
    double rowmax = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
        double r = 0.0;
        for (int j = 0; j < n; ++j) {
            r += fabs(X[i * kE + j]);
        }
        rowmax = fmax(rowmax, r);
    }
    const double norm = block_reduce<NT, true>(sh, c, rowmax);
    int squarings = 0;
    if (norm > 0.5) {
        squarings = max(0, static_cast<int>(ceil(log2(norm / 0.5))));
    }
    const double scale = ldexp(1.0, -squarings);
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e / n, j = e - i * n;
        X[i * kE + j] *= scale;
    }
    __syncthreads();
    // Pade (6,6) coefficients c_k = c_{k-1} (p - k + 1) / (k (2p - k + 1))
    double cf[7];
    cf[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= 6; ++k) {
        cf[k] = cf[k - 1] * static_cast<double>(6 - k + 1) / static_cast<double>(k * (12 - k + 1));
    }
    double *X2 = sh.M[1], *X4 = sh.M[2], *X6 = sh.M[3];
    matmul<NT>(X, X, X2, n);
    matmul<NT>(X2, X2, X4, n);
    matmul<NT>(X4, X2, X6, n);
    // U = c0 + c2 X^2 + c4 X^4 + c6 X^6 (into M[4]); odd factor c1 + c3 X^2 + c5 X^4 (into M[3])
    double *U = sh.M[4], *Vt = sh.M[3];
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e / n, j = e - i * n;
        const double id = i == j ? 1.0 : 0.0;
        const double a = X2[i * kE + j], b = X4[i * kE + j], d = X6[i * kE + j];
        U[i * kE + j] = cf[0] * id + cf[2] * a + cf[4] * b + cf[6] * d;
        Vt[i * kE + j] = cf[1] * id + cf[3] * a + cf[5] * b;
    }
    __syncthreads();
    double *Vo = sh.M[1];
    matmul<NT>(X, Vt, Vo, n); // odd part
    // P = U + Vo (M[5]), Q = U - Vo (M[6])
    double *P = sh.M[5], *Q = sh.M[6];
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e / n, j = e - i * n;
        const double u = U[i * kE + j], v = Vo[i * kE + j];
        P[i * kE + j] = u + v;
        Q[i * kE + j] = u - v;
    }
    __syncthreads();
    // [Q | P] ping-pongs between M[0..1] and M[2..3]; F lands in M[4]
    double *F = sh.M[4];
    gauss_jordan<NT>(Q, P, sh.M[0], sh.M[2], F, n);
    double *spare = sh.M[0];
    for (int s = 0; s < squarings; ++s) {
        matmul<NT>(F, F, spare, n);
        double *t = F;
        F = spare;
        spare = t;
    }
    return F;
}

// two significant digits, rounded up (Expokit's step rounding)
__device__ double round_step(double step) {
    const double s = pow(10.0, floor(log10(step)) - 1.0);
    return ceil(step / s) * s;
}

struct Counters {
    std::int64_t substeps = 0, applies = 0;
};

// c.w (n slots) <- exp(t Q) c.w; returns 0, or an FspOutcome status
template <int NT>
__device__ int expv(Shared &sh, Ctx &c, int n, int m, double t, double tol, Counters &cnt) {
    if (n == 0 || t == 0.0) {
        return 0;
    }
    const int R = c.in->R;
    double rowmax = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        double r = c.diag[k];
        for (int q = 0; q < R; ++q) {
            r += c.coef[q * c.es + k];
        }
        rowmax = fmax(rowmax, r);
    }
    ++cnt.applies;
    const double anorm = fmax(block_reduce<NT, true>(sh, c, rowmax), 1e-300);
    constexpr int max_reject = 10;
    constexpr double btol = 1e-7, gamma = 0.9, delta = 1.2;
    const double t_out = fabs(t), sgn = t < 0.0 ? -1.0 : 1.0;
    double sq0 = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        sq0 += c.w[k] * c.w[k];
    }
    double beta = sqrt(block_reduce<NT, false>(sh, c, sq0));
    if (!(beta > 0.0)) {
        return 0;
    }
    const double fact =
        pow((m + 1) / exp(1.0), m + 1) * sqrt(2.0 * 3.14159265358979323846 * (m + 1));
    double t_new = (1.0 / anorm) * pow((fact * tol) / (4.0 * beta * anorm), 1.0 / m);
    t_new = round_step(t_new);
    double t_now = 0.0;
    for (int sub = 0; t_now < t_out; ++sub) {
        if (sub >= kSubstepLimit) {
            return 2;
        }
        ++cnt.substeps;
        double t_step = fmin(t_out - t_now, t_new);
        const int hd = m + 2;
        for (int e = threadIdx.x; e < hd * hd; e += NT) {
            sh.H[(e / hd) * kE + (e % hd)] = 0.0;
        }
        int k1 = 2, mb = m;
        const double *src = c.w;
        double div = beta;
        double *out = c.buf0;
        for (int j = 0; j < m; ++j) {
            arnoldi_apply<NT>(sh, c, n, src, div, j, out);
            arnoldi_reorthogonalise<NT>(sh, c, n, j + 1, out);
            if (threadIdx.x < 32 && static_cast<int>(threadIdx.x) <= j) {
                sh.H[threadIdx.x * kE + j] = sh.h1[threadIdx.x] + sh.hw[0][threadIdx.x];
            }
            const double s = sqrt(arnoldi_finish<NT>(sh, c, n, j + 1, out));
            ++cnt.applies;
            if (!(s == s)) {
                return 3;
            }
            if (s < btol) {
                k1 = 0;
                mb = j + 1;
                t_step = t_out - t_now;
                break;
            }
            if (threadIdx.x == 0) {
                sh.H[(j + 1) * kE + j] = s;
            }
            src = out;
            div = s;
            out = out == c.buf0 ? c.buf1 : c.buf0;
        }
        double avnorm = 0.0;
        if (k1 != 0) {
            // V_m = src / div, and ||Q V_m||
            double *Vm = c.V + m * c.vs;
            double sq = 0.0;
            for (int k = threadIdx.x; k < n; k += NT) {
                const double y = row(c, R, k, src) / div;
                Vm[k] = src[k] / div;
                sq += y * y;
            }
            ++cnt.applies;
            if (threadIdx.x == 0) {
                sh.H[(m + 1) * kE + m] = 1.0;
            }
            avnorm = sqrt(block_reduce<NT, false>(sh, c, sq));
        } else {
            __syncthreads();
        }
        double err_loc = 0.0, xm = 1.0 / m;
        const double *F = nullptr;
        for (int reject = 0;; ++reject) {
            const int mx = mb + k1;
            for (int e = threadIdx.x; e < mx * mx; e += NT) {
                const int i = e / mx, j = e % mx;
                sh.M[0][i * kE + j] = sgn * t_step * sh.H[i * kE + j];
            }
            __syncthreads();
            F = small_expm<NT>(sh, c, mx);
            if (k1 == 0) {
                err_loc = btol;
                break;
            }
            const double phi1 = fabs(beta * F[m * kE]);
            const double phi2 = fabs(beta * F[(m + 1) * kE] * avnorm);
            if (phi1 > 10.0 * phi2) {
                err_loc = phi2;
                xm = 1.0 / m;
            } else if (phi1 > phi2) {
                err_loc = (phi1 * phi2) / (phi1 - phi2);
                xm = 1.0 / m;
            } else {
                err_loc = phi1;
                xm = 1.0 / max(m - 1, 1);
            }
            if (err_loc <= delta * t_step * tol) {
                break;
            }
            if (reject == max_reject) {
                return 1;
            }
            t_step = gamma * t_step * pow(t_step * tol / err_loc, xm);
            t_step = round_step(t_step);
        }
        const int used = mb + max(0, k1 - 1);
        double sq = 0.0;
        for (int k = threadIdx.x; k < n; k += NT) {
            double v = 0.0;
            for (int j = 0; j < used; ++j) {
                v += (beta * F[j * kE]) * c.V[j * c.vs + k];
            }
            c.w[k] = v;
            sq += v * v;
        }
        beta = sqrt(block_reduce<NT, false>(sh, c, sq));
        t_now += t_step;
        t_new = gamma * t_step * pow(t_step * tol / fmax(err_loc, 1e-300), xm);
        t_new = round_step(t_new);
        if (!(beta == beta)) {
            return 3;
        }
        if (!(beta > 0.0)) {
            break;
        }
    }
    return 0;
}

// ---- support maintenance --------------------------------------------------------------

// the state reached from slot k by reaction r, if the jump exists, stays in the box and leads
// outside the support
__device__ __forceinline__ bool new_neighbour(const Ctx &c, int k, int r, int &j) {
    const FspInstance &in = *c.in;
    const int i = c.s2b[k];
    if (!(c.rate[static_cast<std::int64_t>(r) * in.box + i] > 0.0)) {
        return false;
    }
    int xi[kFspMaxSpecies];
    coords(in, i, xi);
    bool inside = true;
    j = i;
#pragma unroll
    for (int s = 0; s < kFspMaxSpecies; ++s) {
        if (s < in.S) {
            const int y = xi[s] + in.change[r][s];
            inside = inside && y >= 0 && y <= in.bound[s];
            j += in.change[r][s] * in.stride[s];
        }
    }
    return inside && c.b2s[j] < 0;
}

// when reaction r is a jump out of slot k (rate > 0, no count negative) whose target lies above
// the box's bounds, a state the region box(bounds) keeps out of the support: the species it
// crosses the bounds of, as a bit mask (0 otherwise)
__device__ __forceinline__ int clipped_neighbour(const Ctx &c, int k, int r) {
    const FspInstance &in = *c.in;
    const int i = c.s2b[k];
    if (!(c.rate[static_cast<std::int64_t>(r) * in.box + i] > 0.0)) {
        return 0;
    }
    int xi[kFspMaxSpecies];
    coords(in, i, xi);
    bool valid = true;
    int above = 0;
#pragma unroll
    for (int s = 0; s < kFspMaxSpecies; ++s) {
        if (s < in.S) {
            const int y = xi[s] + in.change[r][s];
            valid = valid && y >= 0;
            above |= y > in.bound[s] ? 1 << s : 0;
        }
    }
    return valid ? above : 0;
}

// add `layers` rings of neighbours inside the box to slots [0, n), in the reference's order;
// returns the new n
template <int NT>
__device__ int expand(Shared &sh, const Ctx &c, int n) {
    const FspInstance &in = *c.in;
    const int R = in.R;
    int f0 = 0, f1 = n;
    for (int layer = 0; layer < in.layers && R > 0; ++layer) {
        // candidate q = (slot - f0) * R + r; a state's first discoverer has the smallest q
        const int L = (f1 - f0) * R;
        for (int q = threadIdx.x; q < L; q += NT) {
            int j;
            if (new_neighbour(c, f0 + q / R, q % R, j)) {
                atomicMin(&c.owner[j], q);
            } else if (const int mask = clipped_neighbour(c, f0 + q / R, q % R)) {
                atomicOr(&sh.clipped, mask);
            }
        }
        __syncthreads();
        const int added = compact<NT>(
            sh, L,
            [&](int q) {
                int j;
                return new_neighbour(c, f0 + q / R, q % R, j) && c.owner[j] == q;
            },
            [&](int q, int dest) {
                int j;
                new_neighbour(c, f0 + q / R, q % R, j);
                const int slot = f1 + dest;
                c.b2s[j] = slot;
                c.s2b[slot] = j;
                c.prob[slot] = 0.0;
            });
        for (int slot = f1 + static_cast<int>(threadIdx.x); slot < f1 + added; slot += NT) {
            c.owner[c.s2b[slot]] = kNoOwner;
        }
        __syncthreads();
        f0 = f1;
        f1 += added;
        if (added == 0) {
            break;
        }
    }
    return f1;
}

// ---- adaptive FSP (fsp.hpp:108-188) ---------------------------------------------------------

// the rate out of slot k over every existing jump (the reflecting generator's exit plus leak)
__device__ __forceinline__ double out_rate(const Ctx &c, int k) {
    const FspInstance &in = *c.in;
    const int i = c.s2b[k];
    int xi[kFspMaxSpecies];
    coords(in, i, xi);
    double out = 0.0;
    for (int r = 0; r < in.R; ++r) {
        bool valid = true;
#pragma unroll
        for (int s = 0; s < kFspMaxSpecies; ++s) {
            if (s < in.S) {
                valid = valid && xi[s] + in.change[r][s] >= 0;
            }
        }
        const double a = c.rate[static_cast<std::int64_t>(r) * in.box + i];
        if (a > 0.0 && valid) {
            out += a;
        }
    }
    return out;
}

// probabilities are non-negative: their bit patterns order like the values (-0 counts as 0)
__device__ __forceinline__ unsigned long long prob_key(double p) {
    return p > 0.0 ? static_cast<unsigned long long>(__double_as_longlong(p)) : 0ULL;
}

// flag[k] = 1 for the `count` slots of smallest probability, ties broken by slot (the order of
// num::smallest_indices), else 0: a radix select over the keys, eight bits per pass, then the
// first ties of the selected key in slot order
template <int NT>
__device__ void mark_smallest(Shared &sh, Ctx &c, int n, int count, double *flag) {
    for (int k = threadIdx.x; k < n; k += NT) {
        flag[k] = 0.0;
    }
    __syncthreads();
    if (count <= 0) {
        return;
    }
    unsigned long long prefix = 0ULL;
    int want = count; // rank of the key sought within the keys that share the prefix so far
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += NT) {
            sh.hist[b] = 0;
        }
        __syncthreads();
        const unsigned long long high = shift == 56 ? 0ULL : (~0ULL << (shift + 8));
        for (int k = threadIdx.x; k < n; k += NT) {
            const unsigned long long key = prob_key(c.prob[k]);
            if ((key & high) == (prefix & high)) {
                atomicAdd(&sh.hist[(key >> shift) & 255ULL], 1);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0, b = 0;
            for (; b < 255 && acc + sh.hist[b] < want; ++b) {
                acc += sh.hist[b];
            }
            sh.key = prefix | (static_cast<unsigned long long>(b) << shift);
            sh.i[4] = want - acc;
        }
        __syncthreads();
        prefix = sh.key;
        want = sh.i[4];
        __syncthreads();
    }
    compact<NT>(
        sh, n, [&](int k) { return prob_key(c.prob[k]) == prefix; },
        [&](int k, int dest) {
            if (dest < want) {
                flag[k] = 1.0;
            }
        });
    for (int k = threadIdx.x; k < n; k += NT) {
        if (prob_key(c.prob[k]) < prefix) {
            flag[k] = 1.0;
        }
    }
    __syncthreads();
}

// keep the slots with keep(k), in order, and renormalise to total probability one
template <int NT, typename Keep>
__device__ int keep_and_normalise(Shared &sh, Ctx &c, int n, Keep keep) {
    const int kept = compact<NT>(sh, n, keep, [&](int k, int dest) {
        c.buf0[dest] = c.prob[k];
        c.itmp[dest] = c.s2b[k];
    });
    for (int k = threadIdx.x; k < n; k += NT) {
        c.b2s[c.s2b[k]] = -1;
    }
    __syncthreads();
    double tot = 0.0;
    for (int k = threadIdx.x; k < kept; k += NT) {
        const int j = c.itmp[k];
        c.s2b[k] = j;
        c.b2s[j] = k;
        c.prob[k] = c.buf0[k];
        tot += c.buf0[k];
    }
    const double total = block_reduce<NT, false>(sh, c, tot);
    if (total > 0.0) {
        for (int k = threadIdx.x; k < kept; k += NT) {
            c.prob[k] /= total;
        }
    }
    __syncthreads();
    return kept;
}

template <int NT>
__global__ void __launch_bounds__(NT, 384 / NT + 1) fsp_kernel(const FspBatchView v) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
    Ctx c;
    c.cap = v.cap;
    c.in = &sh.in;
    c.arena = smem_raw + ((sizeof(Shared) + 15) & ~std::size_t(15));
    c.arena_bytes = v.arena_bytes;
    c.parity = 0;
    double *wb = v.work + static_cast<std::int64_t>(blockIdx.x) * fsp_work_doubles(v.cap, v.rmax);
    c.gV = wb;
    c.prob = wb + kBasis * v.cap;
    c.gw = c.prob + v.cap;
    c.gbuf0 = c.gw + v.cap;
    c.gbuf1 = c.gbuf0 + v.cap;
    c.gtmp = c.gbuf1 + v.cap;
    c.gdiag = c.gtmp + v.cap;
    c.gcoef = c.gdiag + v.cap;
    int *ib = v.iwork + static_cast<std::int64_t>(blockIdx.x) * fsp_work_ints(v.cap, v.rmax);
    c.b2s = ib;
    c.s2b = ib + v.cap;
    c.itmp = ib + 2 * v.cap;
    c.owner = ib + 3 * v.cap;
    c.gnbr = ib + 4 * v.cap;

    while (true) {
        if (threadIdx.x == 0) {
            sh.i[1] = atomicAdd(v.queue, 1);
        }
        __syncthreads();
        const int id = sh.i[1];
        if (id >= v.n) {
            return;
        }
        {
            const int *src = reinterpret_cast<const int *>(v.inst + id);
            int *dst = reinterpret_cast<int *>(&sh.in);
            for (int k = threadIdx.x; k < static_cast<int>(sizeof(FspInstance) / 4); k += NT) {
                dst[k] = src[k];
            }
        }
        __syncthreads();
        const FspInstance &in = sh.in;
        c.rate = v.rates + in.rate_offset;
        for (int j = threadIdx.x; j < in.box; j += NT) {
            c.b2s[j] = -1;
            c.owner[j] = kNoOwner;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            c.b2s[in.initial] = 0;
            c.s2b[0] = in.initial;
            c.prob[0] = 1.0;
            sh.clipped = 0;
        }
        __syncthreads();
        int n = 1;
        double t = 0.0, tau = in.initial_step;
        std::int64_t attempt = 0, accepted = 0;
        Counters cnt;
        int status = 0;
        const std::int64_t limit = in.max_steps < kAttemptLimit ? in.max_steps : kAttemptLimit;
        // adaptive FSP: every step is taken (fsp.hpp:133-181)
        for (; in.method == 1 && t < in.final_time && attempt < limit; ++attempt) {
            n = expand<NT>(sh, c, n);
            const int m = min(max(in.krylov_dim, 1), n);
            place(c, n, m);
            double act = 0.0;
            for (int k = threadIdx.x; k < n; k += NT) {
                c.w[k] = c.prob[k];
            }
            assemble<NT>(c, n, true);
            for (int k = threadIdx.x; k < n; k += NT) {
                act += c.prob[k] * c.diag[k];
            }
            const double activity = block_reduce<NT, false>(sh, c, act);
            const double dt = activity > 0.0 ? fmin(in.step_scale / activity, in.final_time - t)
                                             : in.final_time - t;
            status = expv<NT>(sh, c, n, m, dt, in.krylov_tol, cnt);
            if (status != 0) {
                break;
            }
            for (int k = threadIdx.x; k < n; k += NT) {
                c.prob[k] = fmax(0.0, c.w[k]);
            }
            __syncthreads();
            // prune the unlikely states whose probability flux is negligible
            double *drop = c.buf1;
            if (n > 1) {
                double fl = 0.0;
                for (int k = threadIdx.x; k < n; k += NT) {
                    c.tmp[k] = c.prob[k] * out_rate(c, k);
                    fl += c.tmp[k];
                }
                const double total_flux = block_reduce<NT, false>(sh, c, fl);
                const int candidates = min(static_cast<int>(llround(in.prune_fraction * static_cast<double>(n))), n - 1);
                mark_smallest<NT>(sh, c, n, candidates, drop);
                for (int k = threadIdx.x; k < n; k += NT) {
                    const bool d = (drop[k] != 0.0 && c.tmp[k] < in.flux_tolerance * total_flux) ||
                                   c.prob[k] < in.min_probability;
                    drop[k] = d ? 1.0 : 0.0;
                }
            } else {
                for (int k = threadIdx.x; k < n; k += NT) {
                    drop[k] = 0.0;
                }
            }
            __syncthreads();
            n = keep_and_normalise<NT>(sh, c, n, [&](int k) { return drop[k] == 0.0; });
            t += dt;
            ++accepted;
        }
        for (; in.method == 0 && t < in.final_time && attempt < limit; ++attempt) {
            tau = fmin(tau, in.final_time - t);
            n = expand<NT>(sh, c, n);
            const int m = min(max(in.krylov_dim, 1), n);
            place(c, n, m);
            for (int k = threadIdx.x; k < n; k += NT) {
                c.w[k] = c.prob[k];
            }
            assemble<NT>(c, n);
            status = expv<NT>(sh, c, n, m, tau, in.krylov_tol, cnt);
            if (status != 0) {
                break;
            }
            double pos = 0.0;
            for (int k = threadIdx.x; k < n; k += NT) {
                pos += fmax(0.0, c.w[k]);
            }
            const double mass = block_reduce<NT, false>(sh, c, pos);
            if (mass < 1.0 - (in.tolerance * (t + tau) / in.final_time) && tau > 1e-14) {
                tau *= 0.5;
                continue;
            }
            // dp = Q w; keep max(0, w); drop what is both unlikely and nearly constant
            for (int k = threadIdx.x; k < n; k += NT) {
                c.tmp[k] = row(c, in.R, k, c.w);
                c.prob[k] = fmax(0.0, c.w[k]);
            }
            ++cnt.applies;
            __syncthreads();
            const int kept = compact<NT>(
                sh, n,
                [&](int k) {
                    return !(c.prob[k] < in.drop_probability &&
                             fabs(c.tmp[k]) < in.drop_derivative);
                },
                [&](int k, int dest) {
                    c.buf0[dest] = c.prob[k];
                    c.itmp[dest] = c.s2b[k];
                });
            for (int k = threadIdx.x; k < n; k += NT) {
                c.b2s[c.s2b[k]] = -1;
            }
            __syncthreads();
            double tot = 0.0;
            for (int k = threadIdx.x; k < kept; k += NT) {
                const int j = c.itmp[k];
                c.s2b[k] = j;
                c.b2s[j] = k;
                c.prob[k] = c.buf0[k];
                tot += c.buf0[k];
            }
            n = kept;
            const double total = block_reduce<NT, false>(sh, c, tot);
            if (total > 0.0) {
                for (int k = threadIdx.x; k < n; k += NT) {
                    c.prob[k] /= total;
                }
            }
            __syncthreads();
            t += tau;
            ++accepted;
            tau = fmin(tau * in.step_growth, in.final_time - t);
        }
        if (status == 0 && t < in.final_time) {
            status = 2;
        }
        double *out = v.out + in.out_offset;
        for (int j = threadIdx.x; j < in.box; j += NT) {
            out[j] = 0.0;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += NT) {
            out[c.s2b[k]] = c.prob[k];
        }
        if (threadIdx.x == 0) {
            FspOutcome o;
            o.time = t;
            o.attempts = attempt;
            o.accepted = accepted;
            o.support = n;
            o.substeps = cnt.substeps;
            o.applies = cnt.applies;
            o.status = status;
            o.clipped = sh.clipped;
            v.outcome[in.index] = o;
        }
        __syncthreads();
    }
}

constexpr std::size_t kFixedShared = (sizeof(Shared) + 15) & ~std::size_t(15);

template <int NT>
cudaError_t launch_shape(const FspBatchView &v, int blocks, cudaStream_t stream) {
    const std::size_t smem = kFixedShared + v.arena_bytes;
    cudaError_t e = cudaFuncSetAttribute(fsp_kernel<NT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) {
        return e;
    }
    count_launches(1);
    fsp_kernel<NT><<<blocks, NT, smem, stream>>>(v);
    return cudaGetLastError();
}

template <int NT>
int occupancy(std::size_t arena) {
    const std::size_t smem = kFixedShared + arena;
    if (cudaFuncSetAttribute(fsp_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess) {
        return 0;
    }
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fsp_kernel<NT>, NT, smem) !=
        cudaSuccess) {
        return 0;
    }
    return blocks;
}

int occupancy_of(int threads, std::size_t arena) {
    switch (threads) {
    case 128:
        return occupancy<128>(arena);
    case 256:
        return occupancy<256>(arena);
    case 512:
        return occupancy<512>(arena);
    default:
        return 0;
    }
}

} // namespace

std::size_t fsp_fixed_shared_bytes() { return kFixedShared; }

int fsp_blocks_per_sm(int threads) { return occupancy_of(threads, 0); }

std::size_t fsp_arena_bytes(int threads, int blocks_per_sm) {
    if (blocks_per_sm < 1 || occupancy_of(threads, 0) < blocks_per_sm) {
        return 0;
    }
    int dev = 0, per_sm = 0, per_block = 0, reserved = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) !=
            cudaSuccess) {
        return 0;
    }
    std::size_t share = static_cast<std::size_t>(per_sm) / blocks_per_sm;
    share = share > static_cast<std::size_t>(reserved) ? share - reserved : 0;
    share = share < static_cast<std::size_t>(per_block) ? share : per_block;
    std::size_t arena = share > kFixedShared ? (share - kFixedShared) & ~std::size_t(1023) : 0;
    // step down until the occupancy calculator agrees
    while (arena > 0 && occupancy_of(threads, arena) < blocks_per_sm) {
        arena = arena > 4096 ? arena - 4096 : 0;
    }
    return arena;
}

cudaError_t launch_fsp_batch(const FspBatchView &v, int threads, int blocks,
                             cudaStream_t stream) {
    if (blocks <= 0) {
        return cudaErrorInvalidValue;
    }
    switch (threads) {
    case 128:
        return launch_shape<128>(v, blocks, stream);
    case 256:
        return launch_shape<256>(v, blocks, stream);
    case 512:
        return launch_shape<512>(v, blocks, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

} // namespace mkb
