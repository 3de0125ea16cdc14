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
// The support is a compact list of slots with a box-to-slot map, in the reference's order: an
// expansion ring appends the new states in the order the reference discovers them (support
// slot, then reaction; the first discoverer of a state wins, found with an atomic minimum over
// candidate numbers), and dropped states are compacted out in order. Vectors and reductions
// cost the support's size, not the box's.
// One Arnoldi step is three block-wide phases: (1) the operator apply, which also writes the
// basis vector V_j = p / ||p|| of the previous step and accumulates the first Gram-Schmidt
// projections <V_i, Q V_j>; (2) the first subtraction fused with the second projections;
// (3) the second subtraction fused with the norm. The small exponential's elimination runs on
// two warps under a named barrier while the rest of the block waits once.
// Every loop is bounded; no thread waits on another block.
#include "fsp.cuh"
#include "launch_count.hpp"

#include <cmath>

namespace mkb {

namespace {

constexpr int kMaxWarps = 16;
constexpr int kBasis = kFspMaxKrylov + 1;
constexpr int kE = 32;               // side of the small dense matrices in shared memory
constexpr int kDotChunk = 16;        // basis vectors per projection pass
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

// barrier 1 over the first two warps only
__device__ __forceinline__ void pair_barrier() { asm volatile("bar.sync 1, 64;" ::: "memory"); }

struct Shared {
    FspInstance in;
    double H[kE * kE];
    double X[kE * kE], P[kE * kE], Q[kE * kE], PW[kE * kE], T[kE * kE], F[kE * kE];
    double red[kMaxWarps * kE];
    double h1[kE], h2[kE];
    double fac[kE];
    double s[8];
    int i[8];
    int scan[kMaxWarps + 1];
};

// the block's sum (or max) of v, returned to all threads; fixed order, so reproducible
template <int NT, bool MAX>
__device__ double block_reduce(Shared &sh, double v) {
    constexpr int W = NT / 32;
    v = MAX ? warp_max(v) : warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh.red[warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
        double t = lane < W ? sh.red[lane] : (MAX ? -INFINITY : 0.0);
        t = MAX ? warp_max(t) : warp_sum(t);
        if (lane == 0) {
            sh.s[7] = t;
        }
    }
    __syncthreads();
    const double r = sh.s[7];
    __syncthreads();
    return r;
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

struct Ctx {
    const FspInstance *in; // the block's shared copy
    const double *rate;
    double *V;             // kBasis vectors of stride cap
    double *prob, *w, *buf0, *buf1, *tmp;
    int *b2s, *s2b, *itmp, *owner;
    std::int64_t cap;
};

__device__ __forceinline__ void coords(const FspInstance &in, int i, int (&x)[kFspMaxSpecies]) {
#pragma unroll
    for (int s = 0; s < kFspMaxSpecies; ++s) {
        x[s] = s < in.S ? (i / in.stride[s]) % (in.bound[s] + 1) : 0;
    }
}

// Row k of Q applied to src: sum of in-jumps from supported states minus exit * src[k], or
// with ABS the row's absolute sum (src unused). Every valid positive jump counts in the exit.
template <bool ABS>
__device__ __forceinline__ double row_apply(const Ctx &c, int k, const double *src) {
    const FspInstance &in = *c.in;
    const int i = c.s2b[k];
    int xi[kFspMaxSpecies];
    coords(in, i, xi);
    double acc = 0.0, ex = 0.0;
    for (int r = 0; r < in.R; ++r) {
        bool valid = true, inside = true;
        int j = i;
#pragma unroll
        for (int s = 0; s < kFspMaxSpecies; ++s) {
            if (s < in.S) {
                const int ch = in.change[r][s];
                valid = valid && xi[s] + ch >= 0;
                const int xs = xi[s] - ch;
                inside = inside && xs >= 0 && xs <= in.bound[s];
                j -= ch * in.stride[s];
            }
        }
        const double a = c.rate[static_cast<std::int64_t>(r) * in.box + i];
        if (a > 0.0 && valid) {
            ex += a;
        }
        if (inside) {
            const int sl = c.b2s[j];
            if (sl >= 0) {
                const double aj = c.rate[static_cast<std::int64_t>(r) * in.box + j];
                if (aj > 0.0) {
                    if constexpr (ABS) {
                        acc += aj;
                    } else {
                        acc += aj * src[sl];
                    }
                }
            }
        }
    }
    if constexpr (ABS) {
        return acc + ex;
    } else {
        return acc - ex * src[k];
    }
}

// out = Q src over the n slots
template <int NT>
__device__ void apply_plain(const Ctx &c, int n, const double *src, double *out) {
    for (int k = threadIdx.x; k < n; k += NT) {
        out[k] = row_apply<false>(c, k, src);
    }
    __syncthreads();
}

// warp partial sums of acc[q] (basis vector k0 + q, below K) into sh.red
__device__ __forceinline__ void stash_partials(Shared &sh, const double (&acc)[kDotChunk], int k0,
                                               int K) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < kDotChunk; ++q) {
        if (k0 + q < K) {
            const double v = warp_sum(acc[q]);
            if (lane == 0) {
                sh.red[warp * kE + k0 + q] = v;
            }
        }
    }
}

// h[i] = sum over warps of the stashed partials, i < K, visible to every thread on return
template <int NT>
__device__ void finish_dots(Shared &sh, int K, double *h) {
    constexpr int W = NT / 32;
    __syncthreads();
    if (static_cast<int>(threadIdx.x) < K) {
        double t = 0.0;
        for (int w = 0; w < W; ++w) {
            t += sh.red[w * kE + threadIdx.x];
        }
        h[threadIdx.x] = t;
    }
    __syncthreads();
}

__device__ __forceinline__ void zero(double (&acc)[kDotChunk]) {
#pragma unroll
    for (int q = 0; q < kDotChunk; ++q) {
        acc[q] = 0.0;
    }
}

// Arnoldi phase 1: V_j = src / div, out = Q V_j, sh.h1[i] = <V_i, out> for i <= j
template <int NT>
__device__ void arnoldi_apply(Shared &sh, const Ctx &c, int n, const double *src, double div,
                              int j, double *out) {
    const int K = j + 1;
    double *Vj = c.V + static_cast<std::int64_t>(j) * c.cap;
    double acc[kDotChunk];
    zero(acc);
    for (int k = threadIdx.x; k < n; k += NT) {
        const double y = row_apply<false>(c, k, src) / div;
        const double vk = src[k] / div;
        Vj[k] = vk;
        out[k] = y;
#pragma unroll
        for (int q = 0; q < kDotChunk; ++q) {
            if (q < K) {
                const double v = q == j ? vk : c.V[q * c.cap + k];
                acc[q] += v * y;
            }
        }
    }
    stash_partials(sh, acc, 0, K);
    for (int k0 = kDotChunk; k0 < K; k0 += kDotChunk) {
        zero(acc);
        for (int k = threadIdx.x; k < n; k += NT) {
            const double y = out[k];
#pragma unroll
            for (int q = 0; q < kDotChunk; ++q) {
                if (k0 + q < K) {
                    acc[q] += c.V[(k0 + q) * c.cap + k] * y;
                }
            }
        }
        stash_partials(sh, acc, k0, K);
    }
    finish_dots<NT>(sh, K, sh.h1);
}

// Arnoldi phase 2: out -= sum_i h1[i] V_i, then sh.h2[i] = <V_i, out>
template <int NT>
__device__ void arnoldi_reorthogonalise(Shared &sh, const Ctx &c, int n, int K, double *out) {
    double acc[kDotChunk];
    zero(acc);
    for (int k = threadIdx.x; k < n; k += NT) {
        double v = out[k];
        for (int i = 0; i < K; ++i) {
            v -= sh.h1[i] * c.V[i * c.cap + k];
        }
        out[k] = v;
#pragma unroll
        for (int q = 0; q < kDotChunk; ++q) {
            if (q < K) {
                acc[q] += c.V[q * c.cap + k] * v;
            }
        }
    }
    stash_partials(sh, acc, 0, K);
    for (int k0 = kDotChunk; k0 < K; k0 += kDotChunk) {
        zero(acc);
        for (int k = threadIdx.x; k < n; k += NT) {
            const double v = out[k];
#pragma unroll
            for (int q = 0; q < kDotChunk; ++q) {
                if (k0 + q < K) {
                    acc[q] += c.V[(k0 + q) * c.cap + k] * v;
                }
            }
        }
        stash_partials(sh, acc, k0, K);
    }
    finish_dots<NT>(sh, K, sh.h2);
}

// Arnoldi phase 3: out -= sum_i h2[i] V_i; returns ||out||^2
template <int NT>
__device__ double arnoldi_finish(Shared &sh, const Ctx &c, int n, int K, double *out) {
    double sq = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        double v = out[k];
        for (int i = 0; i < K; ++i) {
            v -= sh.h2[i] * c.V[i * c.cap + k];
        }
        out[k] = v;
        sq += v * v;
    }
    return block_reduce<NT, false>(sh, sq);
}

template <int NT>
__device__ double dot(Shared &sh, const double *a, const double *b, int n) {
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        v += a[k] * b[k];
    }
    return block_reduce<NT, false>(sh, v);
}

// C = A B for n x n matrices in shared memory (row-major, side kE)
template <int NT>
__device__ void matmul(const double *A, const double *B, double *C, int n) {
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e / n, j = e % n;
        double s = 0.0;
        for (int k = 0; k < n; ++k) {
            s += A[i * kE + k] * B[k * kE + j];
        }
        C[i * kE + j] = s;
    }
    __syncthreads();
}

// F = Q^{-1} F by Gauss-Jordan elimination with partial pivoting (first largest pivot), on the
// first two warps: thread j < 32 owns column j of Q, thread 32 + j column j of F. The pivot
// row is swapped in by each column's owner; the factors come from warp 0 before the swap.
template <int NT>
__device__ void solve_pade(Shared &sh, int n) {
    if (threadIdx.x < 64) {
        const int lane = threadIdx.x & 31;
        double *M = threadIdx.x < 32 ? sh.Q : sh.F;
        for (int k = 0; k < n; ++k) {
            if (threadIdx.x < 32) {
                double a = (lane >= k && lane < n) ? fabs(sh.Q[lane * kE + k]) : -1.0;
                int idx = lane;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const double oa = __shfl_xor_sync(0xffffffffu, a, off);
                    const int oi = __shfl_xor_sync(0xffffffffu, idx, off);
                    if (oa > a || (oa == a && oi < idx)) {
                        a = oa;
                        idx = oi;
                    }
                }
                const int piv = idx;
                const double pivot = sh.Q[piv * kE + k];
                if (lane < n) {
                    const int src = lane == k ? piv : (lane == piv ? k : lane);
                    sh.fac[lane] = lane == k ? 0.0 : sh.Q[src * kE + k] / pivot;
                }
                if (lane == 0) {
                    sh.i[0] = piv;
                }
            }
            pair_barrier();
            const int piv = sh.i[0];
            if (lane < n) {
                const double rk = M[piv * kE + lane];
                M[piv * kE + lane] = M[k * kE + lane];
                M[k * kE + lane] = rk;
                for (int i = 0; i < n; ++i) {
                    const double f = sh.fac[i];
                    if (f != 0.0) {
                        M[i * kE + lane] -= f * rk;
                    }
                }
            }
            pair_barrier();
        }
        if (threadIdx.x >= 32 && lane < n) {
            for (int i = 0; i < n; ++i) {
                sh.F[i * kE + lane] /= sh.Q[i * kE + i];
            }
        }
    }
    __syncthreads();
}

// sh.F = exp(sh.X) for an n x n matrix: Pade (6,6) with scaling and squaring
template <int NT>
__device__ void small_expm(Shared &sh, int n) {
    double rowmax = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
        double r = 0.0;
        for (int j = 0; j < n; ++j) {
            r += fabs(sh.X[i * kE + j]);
        }
        rowmax = fmax(rowmax, r);
    }
    const double norm = block_reduce<NT, true>(sh, rowmax);
    int squarings = 0;
    if (norm > 0.5) {
        squarings = max(0, static_cast<int>(ceil(log2(norm / 0.5))));
    }
    const double scale = ldexp(1.0, -squarings);
    for (int e = threadIdx.x; e < n * n; e += NT) {
        const int i = e / n, j = e % n;
        sh.X[i * kE + j] *= scale;
        const double id = i == j ? 1.0 : 0.0;
        sh.PW[i * kE + j] = id;
        sh.P[i * kE + j] = id;
        sh.Q[i * kE + j] = id;
    }
    __syncthreads();
    constexpr int p = 6;
    double cf = 1.0;
    for (int k = 1; k <= p; ++k) {
        cf *= static_cast<double>(p - k + 1) / static_cast<double>(k * ((2 * p) - k + 1));
        matmul<NT>(sh.PW, sh.X, sh.T, n);
        const double sign = (k % 2 == 0) ? 1.0 : -1.0;
        for (int e = threadIdx.x; e < n * n; e += NT) {
            const int i = e / n, j = e % n;
            const double v = sh.T[i * kE + j];
            sh.PW[i * kE + j] = v;
            sh.P[i * kE + j] += cf * v;
            sh.Q[i * kE + j] += sign * cf * v;
            if (k == p) {
                sh.F[i * kE + j] = sh.P[i * kE + j];
            }
        }
        __syncthreads();
    }
    solve_pade<NT>(sh, n);
    for (int s = 0; s < squarings; ++s) {
        matmul<NT>(sh.F, sh.F, sh.T, n);
        for (int e = threadIdx.x; e < n * n; e += NT) {
            const int i = e / n, j = e % n;
            sh.F[i * kE + j] = sh.T[i * kE + j];
        }
        __syncthreads();
    }
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
__device__ int expv(Shared &sh, const Ctx &c, int n, double t, int m_req, double tol,
                    Counters &cnt) {
    if (n == 0 || t == 0.0) {
        return 0;
    }
    const int m = min(max(m_req, 1), n);
    double rowmax = 0.0;
    for (int k = threadIdx.x; k < n; k += NT) {
        rowmax = fmax(rowmax, row_apply<true>(c, k, nullptr));
    }
    ++cnt.applies;
    const double anorm = fmax(block_reduce<NT, true>(sh, rowmax), 1e-300);
    constexpr int max_reject = 10;
    constexpr double btol = 1e-7, gamma = 0.9, delta = 1.2;
    const double t_out = fabs(t), sgn = t < 0.0 ? -1.0 : 1.0;
    double beta = sqrt(dot<NT>(sh, c.w, c.w, n));
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
        __syncthreads();
        int k1 = 2, mb = m;
        const double *src = c.w;
        double div = beta;
        double *out = c.buf0;
        for (int j = 0; j < m; ++j) {
            arnoldi_apply<NT>(sh, c, n, src, div, j, out);
            arnoldi_reorthogonalise<NT>(sh, c, n, j + 1, out);
            for (int i = threadIdx.x; i <= j; i += NT) {
                sh.H[i * kE + j] = sh.h1[i] + sh.h2[i];
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
            double *Vm = c.V + static_cast<std::int64_t>(m) * c.cap;
            double sq = 0.0;
            for (int k = threadIdx.x; k < n; k += NT) {
                const double y = row_apply<false>(c, k, src) / div;
                Vm[k] = src[k] / div;
                sq += y * y;
            }
            ++cnt.applies;
            if (threadIdx.x == 0) {
                sh.H[(m + 1) * kE + m] = 1.0;
            }
            avnorm = sqrt(block_reduce<NT, false>(sh, sq));
        }
        double err_loc = 0.0, xm = 1.0 / m;
        for (int reject = 0;; ++reject) {
            const int mx = mb + k1;
            for (int e = threadIdx.x; e < mx * mx; e += NT) {
                const int i = e / mx, j = e % mx;
                sh.X[i * kE + j] = sgn * t_step * sh.H[i * kE + j];
            }
            __syncthreads();
            small_expm<NT>(sh, mx);
            if (k1 == 0) {
                err_loc = btol;
                break;
            }
            const double phi1 = fabs(beta * sh.F[m * kE]);
            const double phi2 = fabs(beta * sh.F[(m + 1) * kE] * avnorm);
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
                v += (beta * sh.F[j * kE]) * c.V[static_cast<std::int64_t>(j) * c.cap + k];
            }
            c.w[k] = v;
            sq += v * v;
        }
        beta = sqrt(block_reduce<NT, false>(sh, sq));
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

template <int NT>
__global__ void __launch_bounds__(NT, 384 / NT + 1) fsp_kernel(const FspBatchView v) {
    extern __shared__ double smem_raw[];
    Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
    Ctx c;
    c.cap = v.cap;
    c.in = &sh.in;
    double *wb = v.work + static_cast<std::int64_t>(blockIdx.x) * fsp_work_doubles(v.cap);
    c.V = wb;
    c.prob = wb + kBasis * v.cap;
    c.w = c.prob + v.cap;
    c.buf0 = c.w + v.cap;
    c.buf1 = c.buf0 + v.cap;
    c.tmp = c.buf1 + v.cap;
    int *ib = v.iwork + static_cast<std::int64_t>(blockIdx.x) * fsp_work_ints(v.cap);
    c.b2s = ib;
    c.s2b = ib + v.cap;
    c.itmp = ib + 2 * v.cap;
    c.owner = ib + 3 * v.cap;

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
        }
        __syncthreads();
        int n = 1;
        double t = 0.0, tau = in.initial_step;
        std::int64_t attempt = 0, accepted = 0;
        Counters cnt;
        int status = 0;
        const std::int64_t limit = in.max_steps < kAttemptLimit ? in.max_steps : kAttemptLimit;
        for (; t < in.final_time && attempt < limit; ++attempt) {
            tau = fmin(tau, in.final_time - t);
            n = expand<NT>(sh, c, n);
            for (int k = threadIdx.x; k < n; k += NT) {
                c.w[k] = c.prob[k];
            }
            __syncthreads();
            status = expv<NT>(sh, c, n, tau, in.krylov_dim, in.krylov_tol, cnt);
            if (status != 0) {
                break;
            }
            double pos = 0.0;
            for (int k = threadIdx.x; k < n; k += NT) {
                pos += fmax(0.0, c.w[k]);
            }
            const double mass = block_reduce<NT, false>(sh, pos);
            if (mass < 1.0 - (in.tolerance * (t + tau) / in.final_time) && tau > 1e-14) {
                tau *= 0.5;
                continue;
            }
            // dp = Q w; keep max(0, w); drop what is both unlikely and nearly constant
            apply_plain<NT>(c, n, c.w, c.tmp);
            ++cnt.applies;
            for (int k = threadIdx.x; k < n; k += NT) {
                c.prob[k] = fmax(0.0, c.w[k]);
            }
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
            const double total = block_reduce<NT, false>(sh, tot);
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
            v.outcome[in.index] = o;
        }
        __syncthreads();
    }
}

template <int NT>
cudaError_t launch_shape(const FspBatchView &v, int blocks, cudaStream_t stream) {
    const std::size_t smem = sizeof(Shared);
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
int blocks_per_sm_shape() {
    const std::size_t smem = sizeof(Shared);
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

} // namespace

std::size_t fsp_shared_bytes() { return sizeof(Shared); }

int fsp_blocks_per_sm(int threads) {
    switch (threads) {
    case 128:
        return blocks_per_sm_shape<128>();
    case 256:
        return blocks_per_sm_shape<256>();
    case 512:
        return blocks_per_sm_shape<512>();
    default:
        return 0;
    }
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
