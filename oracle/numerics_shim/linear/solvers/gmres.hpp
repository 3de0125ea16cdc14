// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
//
// Restarted GMRES as MarkovKit calls it: num::gmres(A, b, x, options) and
// num::gmres(A, M, b, x, options) returning {iterations, residual, converged}
// (call sites tests/test_rdme.cpp:238-249, examples/rdme_multigrid_benchmark.cpp:82-104).
// The library source is absent, so its internals are restated from the published method:
// Saad, "Iterative Methods for Sparse Linear Systems", 2nd ed., Alg. 6.9 (GMRES with
// modified Gram-Schmidt Arnoldi and Givens rotations) and Alg. 9.5 (right preconditioning,
// so the monitored residual is the unpreconditioned one). The tolerance is absolute on the
// Euclidean residual norm, as the paper driver uses it (rdme/cpp/rdme_full_multigrid.cpp:1202-1205).
// `iterations` counts Arnoldi steps; `residual` is the recomputed true residual norm.
#pragma once

#include "container/vector.hpp"
#include "linear/operator.hpp"
#include <algorithm>
#include <cmath>

namespace num {

struct gmres_options {
    real tolerance = 1e-8;
    idx max_iterations = 1000;
    idx restart = 30;
};

struct solver_result {
    idx iterations = 0;
    real residual = 0.0;
    bool converged = false;
};

namespace detail {

struct identity_preconditioner {
    [[nodiscard]] idx rows() const { return 0; }
    [[nodiscard]] idx cols() const { return 0; }
    void apply(const vec<real> &x, vec<real> &y) const { y = x; }
};

inline real dot(const vec<real> &a, const vec<real> &b) {
    real s = 0.0;
    for (idx i = 0; i < a.size(); ++i) {
        s += a[i] * b[i];
    }
    return s;
}

inline real norm2(const vec<real> &a) { return std::sqrt(dot(a, a)); }

template <typename Op, typename Pre>
solver_result gmres_impl(const Op &A, const Pre &M, const vec<real> &b, vec<real> &x,
                         const gmres_options &options) {
    const idx n = b.size();
    const idx m = std::max<idx>(1, std::min(options.restart, std::max<idx>(n, 1)));
    if (x.size() != n) {
        x.assign(n, 0.0);
    }
    solver_result result;
    vec<real> r(n), w(n), z(n);
    const auto true_residual = [&]() {
        A.apply(x, w);
        for (idx i = 0; i < n; ++i) {
            r[i] = b[i] - w[i];
        }
        return norm2(r);
    };
    real beta = true_residual();
    result.residual = beta;
    if (beta <= options.tolerance) {
        result.converged = true;
        return result;
    }
    array<vec<real>> V(m + 1, vec<real>(n, 0.0));
    array<vec<real>> H(m + 1, vec<real>(m, 0.0)); // H[i][j]
    vec<real> cs(m, 0.0), sn(m, 0.0), g(m + 1, 0.0), y(m, 0.0);

    while (result.iterations < options.max_iterations) {
        for (idx i = 0; i < n; ++i) {
            V[0][i] = r[i] / beta;
        }
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        idx k = 0; // columns built in this cycle
        bool done = false;
        for (idx j = 0; j < m && result.iterations < options.max_iterations; ++j) {
            M.apply(V[j], z);
            A.apply(z, w);
            for (idx i = 0; i <= j; ++i) {
                H[i][j] = dot(w, V[i]);
                for (idx t = 0; t < n; ++t) {
                    w[t] -= H[i][j] * V[i][t];
                }
            }
            const real h = norm2(w);
            H[j + 1][j] = h;
            for (idx i = 0; i < j; ++i) {
                const real a = H[i][j], c = H[i + 1][j];
                H[i][j] = cs[i] * a + sn[i] * c;
                H[i + 1][j] = -sn[i] * a + cs[i] * c;
            }
            const real a = H[j][j], c = H[j + 1][j];
            const real denom = std::hypot(a, c);
            cs[j] = denom > 0.0 ? a / denom : 1.0;
            sn[j] = denom > 0.0 ? c / denom : 0.0;
            H[j][j] = denom;
            H[j + 1][j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++result.iterations;
            k = j + 1;
            if (std::abs(g[j + 1]) <= options.tolerance || !(h > 0.0)) {
                done = true;
                break;
            }
            for (idx t = 0; t < n; ++t) {
                V[j + 1][t] = w[t] / h;
            }
        }
        // x += M V_k y_k with H_k y_k = g_k
        for (idx i = k; i-- > 0;) {
            real s = g[i];
            for (idx t = i + 1; t < k; ++t) {
                s -= H[i][t] * y[t];
            }
            y[i] = s / H[i][i];
        }
        std::fill(w.begin(), w.end(), 0.0);
        for (idx j = 0; j < k; ++j) {
            for (idx t = 0; t < n; ++t) {
                w[t] += y[j] * V[j][t];
            }
        }
        M.apply(w, z);
        for (idx t = 0; t < n; ++t) {
            x[t] += z[t];
        }
        beta = true_residual();
        result.residual = beta;
        if (beta <= options.tolerance) {
            result.converged = true;
            return result;
        }
        if (done && !(std::abs(g[k]) > 0.0)) {
            // exact breakdown without reaching the tolerance: restart from the true residual
        }
    }
    result.converged = result.residual <= options.tolerance;
    return result;
}

} // namespace detail

template <typename Op>
solver_result gmres(const Op &A, const vec<real> &b, vec<real> &x,
                    const gmres_options &options = {}) {
    return detail::gmres_impl(A, detail::identity_preconditioner{}, b, x, options);
}

template <typename Op, typename Pre>
solver_result gmres(const Op &A, const Pre &M, const vec<real> &b, vec<real> &x,
                    const gmres_options &options = {}) {
    return detail::gmres_impl(A, M, b, x, options);
}

} // namespace num
