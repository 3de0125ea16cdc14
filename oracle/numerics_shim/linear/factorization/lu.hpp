// ORACLE TEST INFRASTRUCTURE — numerics shim (see core/types.hpp).
// Dense LU with partial pivoting; `singular` reports an exactly zero pivot. Used by
// population_multigrid::factor (markovkit/rdme/multigrid.hpp:247-264) and its cycle (:221).
#pragma once

#include "container/matrix.hpp"
#include <cmath>
#include <utility>

namespace num {

template <typename T>
struct lu_result {
    mat<T> factors; // unit lower triangle below the diagonal, upper triangle on and above
    array<idx> pivot;
    bool singular = false;
};

template <typename T>
lu_result<T> lu(mat<T> A) {
    const idx n = A.rows();
    lu_result<T> result;
    result.pivot.resize(n);
    for (idx k = 0; k < n; ++k) {
        idx p = k;
        for (idx i = k + 1; i < n; ++i) {
            if (std::abs(A(i, k)) > std::abs(A(p, k))) {
                p = i;
            }
        }
        result.pivot[k] = p;
        if (p != k) {
            for (idx j = 0; j < n; ++j) {
                std::swap(A(k, j), A(p, j));
            }
        }
        if (A(k, k) == T(0)) {
            result.singular = true;
            continue;
        }
        for (idx i = k + 1; i < n; ++i) {
            A(i, k) /= A(k, k);
            for (idx j = k + 1; j < n; ++j) {
                A(i, j) -= A(i, k) * A(k, j);
            }
        }
    }
    result.factors = std::move(A);
    return result;
}

// x = A^{-1} b from the factors
template <typename T, typename In, typename Out>
void solve(const lu_result<T> &f, const In &b, Out &x) {
    const idx n = f.factors.rows();
    array<T> y(b.begin(), b.begin() + n);
    for (idx k = 0; k < n; ++k) {
        std::swap(y[k], y[f.pivot[k]]);
    }
    for (idx i = 0; i < n; ++i) {
        for (idx j = 0; j < i; ++j) {
            y[i] -= f.factors(i, j) * y[j];
        }
    }
    for (idx i = n; i-- > 0;) {
        for (idx j = i + 1; j < n; ++j) {
            y[i] -= f.factors(i, j) * y[j];
        }
        y[i] /= f.factors(i, i);
    }
    for (idx i = 0; i < n; ++i) {
        x[i] = y[i];
    }
}

} // namespace num
