// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
//
// w = exp(t A) v by Krylov projection, as MarkovKit calls num::expv(t, A, v, m, tol)
// (markovkit/fsp.hpp:152,223; examples/rdme_two_particle_annihilation.cpp:236). The library
// source is absent; this restates Sidje's Expokit `expv` step-size controller (R. B. Sidje,
// ACM TOMS 24(1):130-156, 1998): Arnoldi with m vectors, the augmented (m+2)x(m+2)
// Hessenberg exponential, the two-term local error estimate and the 0.9 / 1.2 safety
// factors. The small exponential uses a diagonal (6,6) Pade approximant with scaling and
// squaring (the method Expokit's DGPADM names).
#pragma once

#include "container/matrix.hpp"
#include "container/vector.hpp"
#include "linear/sparse/sparse.hpp"
#include <algorithm>
#include <cmath>
#include <numbers>
#include <numeric>
#include <stdexcept>

namespace num {

namespace detail {

// exp(A) for a small dense n x n matrix (row-major), Pade (6,6) with scaling and squaring
inline array<real> small_expm(const array<real> &A, idx n) {
    real norm = 0.0;
    for (idx i = 0; i < n; ++i) {
        real s = 0.0;
        for (idx j = 0; j < n; ++j) {
            s += std::abs(A[(i * n) + j]);
        }
        norm = std::max(norm, s);
    }
    int squarings = 0;
    if (norm > 0.5) {
        squarings = std::max(0, static_cast<int>(std::ceil(std::log2(norm / 0.5))));
    }
    const real scale = std::ldexp(1.0, -squarings);
    array<real> X(n * n), P(n * n, 0.0), Q(n * n, 0.0), T(n * n);
    for (idx k = 0; k < n * n; ++k) {
        X[k] = A[k] * scale;
    }
    const auto matmul = [n](const array<real> &a, const array<real> &b, array<real> &c) {
        for (idx i = 0; i < n; ++i) {
            for (idx j = 0; j < n; ++j) {
                real s = 0.0;
                for (idx k = 0; k < n; ++k) {
                    s += a[(i * n) + k] * b[(k * n) + j];
                }
                c[(i * n) + j] = s;
            }
        }
    };
    constexpr int p = 6;
    real c = 1.0;
    array<real> power(n * n, 0.0);
    for (idx i = 0; i < n; ++i) {
        power[(i * n) + i] = 1.0;
    }
    for (int k = 0; k <= p; ++k) {
        if (k > 0) {
            c *= static_cast<real>(p - k + 1) / static_cast<real>(k * ((2 * p) - k + 1));
            matmul(power, X, T);
            power.swap(T);
        }
        const real sign = (k % 2 == 0) ? 1.0 : -1.0;
        for (idx e = 0; e < n * n; ++e) {
            P[e] += c * power[e];
            Q[e] += sign * c * power[e];
        }
    }
    // F = Q^{-1} P by Gaussian elimination with partial pivoting
    array<real> F = P;
    for (idx k = 0; k < n; ++k) {
        idx piv = k;
        for (idx i = k + 1; i < n; ++i) {
            if (std::abs(Q[(i * n) + k]) > std::abs(Q[(piv * n) + k])) {
                piv = i;
            }
        }
        if (piv != k) {
            for (idx j = 0; j < n; ++j) {
                std::swap(Q[(k * n) + j], Q[(piv * n) + j]);
                std::swap(F[(k * n) + j], F[(piv * n) + j]);
            }
        }
        for (idx i = 0; i < n; ++i) {
            if (i == k) {
                continue;
            }
            const real f = Q[(i * n) + k] / Q[(k * n) + k];
            if (f == 0.0) {
                continue;
            }
            for (idx j = 0; j < n; ++j) {
                Q[(i * n) + j] -= f * Q[(k * n) + j];
                F[(i * n) + j] -= f * F[(k * n) + j];
            }
        }
    }
    for (idx i = 0; i < n; ++i) {
        const real d = Q[(i * n) + i];
        for (idx j = 0; j < n; ++j) {
            F[(i * n) + j] /= d;
        }
    }
    for (int s = 0; s < squarings; ++s) {
        matmul(F, F, T);
        F.swap(T);
    }
    return F;
}

template <typename Op>
real operator_norm_estimate(const Op &A) {
    if constexpr (requires { A.norm_inf(); }) {
        return A.norm_inf();
    } else {
        // power iteration on |A|-like growth of a positive vector
        const idx n = A.rows();
        vec<real> x(n, 1.0 / std::sqrt(static_cast<real>(n))), y(n, 0.0);
        real estimate = 0.0;
        for (int it = 0; it < 20; ++it) {
            A.apply(x, y);
            real norm = 0.0;
            for (real v : y) {
                norm += v * v;
            }
            norm = std::sqrt(norm);
            if (!(norm > 0.0)) {
                break;
            }
            estimate = norm;
            for (idx i = 0; i < n; ++i) {
                x[i] = y[i] / norm;
            }
        }
        return estimate;
    }
}

inline real round_step(real step) {
    const real s = std::pow(10.0, std::floor(std::log10(step)) - 1.0);
    return std::ceil(step / s) * s;
}

} // namespace detail

template <typename Op>
vec<real> expv(real t, const Op &A, const vec<real> &v, int m = 30, real tol = 1e-7) {
    const idx n = v.size();
    vec<real> w = v;
    if (n == 0 || t == 0.0) {
        return w;
    }
    m = static_cast<int>(std::min<idx>(static_cast<idx>(std::max(m, 1)), n));
    const real anorm = std::max(detail::operator_norm_estimate(A), 1e-300);
    constexpr int max_reject = 10;
    constexpr real breakdown_tol = 1e-7;
    constexpr real gamma = 0.9;
    constexpr real delta = 1.2;
    const real t_out = std::abs(t);
    const real sgn = t < 0.0 ? -1.0 : 1.0;
    real beta = std::sqrt(std::inner_product(v.begin(), v.end(), v.begin(), 0.0));
    if (!(beta > 0.0)) {
        return w;
    }
    const real fact = std::pow((m + 1) / std::exp(1.0), m + 1) * std::sqrt(2.0 * std::numbers::pi * (m + 1));
    real t_new = (1.0 / anorm) * std::pow((fact * tol) / (4.0 * beta * anorm), 1.0 / m);
    t_new = detail::round_step(t_new);
    real t_now = 0.0;

    array<vec<real>> V(m + 1, vec<real>(n, 0.0));
    vec<real> p(n);
    while (t_now < t_out) {
        real t_step = std::min(t_out - t_now, t_new);
        const idx H_dim = m + 2;
        array<real> H(H_dim * H_dim, 0.0);
        for (idx i = 0; i < n; ++i) {
            V[0][i] = w[i] / beta;
        }
        int k1 = 2, mb = m;
        for (int j = 0; j < m; ++j) {
            A.apply(V[j], p);
            for (int i = 0; i <= j; ++i) {
                real h = 0.0;
                for (idx q = 0; q < n; ++q) {
                    h += V[i][q] * p[q];
                }
                H[(i * H_dim) + j] = h;
                for (idx q = 0; q < n; ++q) {
                    p[q] -= h * V[i][q];
                }
            }
            const real s = std::sqrt(std::inner_product(p.begin(), p.end(), p.begin(), 0.0));
            if (s < breakdown_tol) {
                k1 = 0;
                mb = j + 1;
                t_step = t_out - t_now;
                break;
            }
            H[((j + 1) * H_dim) + j] = s;
            for (idx q = 0; q < n; ++q) {
                V[j + 1][q] = p[q] / s;
            }
        }
        real avnorm = 0.0;
        if (k1 != 0) {
            H[((m + 1) * H_dim) + m] = 1.0;
            A.apply(V[m], p);
            avnorm = std::sqrt(std::inner_product(p.begin(), p.end(), p.begin(), 0.0));
        }
        real err_loc = 0.0;
        real xm = 1.0 / m;
        array<real> F;
        idx mx = 0;
        for (int reject = 0;; ++reject) {
            mx = static_cast<idx>(mb + k1);
            array<real> Hs(mx * mx);
            for (idx i = 0; i < mx; ++i) {
                for (idx j = 0; j < mx; ++j) {
                    Hs[(i * mx) + j] = sgn * t_step * H[(i * H_dim) + j];
                }
            }
            F = detail::small_expm(Hs, mx);
            if (k1 == 0) {
                err_loc = breakdown_tol;
                break;
            }
            const real phi1 = std::abs(beta * F[static_cast<idx>(m) * mx]);
            const real phi2 = std::abs(beta * F[static_cast<idx>(m + 1) * mx] * avnorm);
            if (phi1 > 10.0 * phi2) {
                err_loc = phi2;
                xm = 1.0 / m;
            } else if (phi1 > phi2) {
                err_loc = (phi1 * phi2) / (phi1 - phi2);
                xm = 1.0 / m;
            } else {
                err_loc = phi1;
                xm = 1.0 / std::max(m - 1, 1);
            }
            if (err_loc <= delta * t_step * tol) {
                break;
            }
            if (reject == max_reject) {
                throw std::runtime_error("expv: the requested tolerance is too high");
            }
            t_step = gamma * t_step * std::pow(t_step * tol / err_loc, xm);
            t_step = detail::round_step(t_step);
        }
        const idx used = static_cast<idx>(mb + std::max(0, k1 - 1));
        std::fill(w.begin(), w.end(), 0.0);
        for (idx j = 0; j < used; ++j) {
            const real c = beta * F[j * mx];
            for (idx q = 0; q < n; ++q) {
                w[q] += c * V[j][q];
            }
        }
        beta = std::sqrt(std::inner_product(w.begin(), w.end(), w.begin(), 0.0));
        t_now += t_step;
        t_new = gamma * t_step * std::pow(t_step * tol / std::max(err_loc, 1e-300), xm);
        t_new = detail::round_step(t_new);
        if (!(beta > 0.0)) {
            break;
        }
    }
    return w;
}

} // namespace num
