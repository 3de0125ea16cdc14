"""ORACLE TEST INFRASTRUCTURE — not part of the product; only tests/ import it.

ILU(0) as num::ilu0_preconditioner(A) computes it for MarkovKit's RDME benchmark
(examples/rdme_multigrid_benchmark.cpp:115; the paper drivers call the same factorisation as
num::ilu0_factor(values, ptr, column, diagonal, scratch, n), e.g.
rdme/paper/data/reflection_fsp/current_source.cpp:986). That function lives in the numerics
library, the un-vendored git submodule ext/numerics (github.com/AdityaDendukuri/numerics; its
revision is not recorded in the reference tree), so this restates the published algorithm:
Saad, Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 10.4 (ILU(0), IKJ variant,
with a dense marker of row i's pattern), then forward substitution with the unit lower factor
and backward substitution with the upper one. Parity unpinned: the reference holds no golden
vector for it. Pure-Python loops: small matrices only.
"""

from __future__ import annotations

import numpy as np


def ilu0_factor(ptr: np.ndarray, col: np.ndarray, val: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(lu, diag): L strictly below the diagonal (unit diagonal implied) and U on and above it,
    in A's pattern; diag[i] = position of row i's diagonal. Columns ascending within rows."""
    n = len(ptr) - 1
    lu = np.array(val, dtype=np.float64, copy=True)
    diag = np.full(n, -1, dtype=np.int64)
    for i in range(n):
        for p in range(ptr[i], ptr[i + 1]):
            if col[p] == i:
                diag[i] = p
        if diag[i] < 0:
            raise ValueError(f"row {i} has no diagonal entry")
    marker = np.full(n, -1, dtype=np.int64)
    for i in range(n):
        b, e = int(ptr[i]), int(ptr[i + 1])
        for p in range(b, e):
            marker[col[p]] = p
        for p in range(b, int(diag[i])):
            k = int(col[p])
            lik = lu[p] / lu[diag[k]]
            lu[p] = lik
            for q in range(int(diag[k]) + 1, int(ptr[k + 1])):
                at = marker[col[q]]
                if at >= 0:
                    lu[at] -= lik * lu[q]
        for p in range(b, e):
            marker[col[p]] = -1
    return lu, diag


def ilu0_solve(ptr: np.ndarray, col: np.ndarray, lu: np.ndarray, diag: np.ndarray, v: np.ndarray) -> np.ndarray:
    """z = U^-1 L^-1 v"""
    n = len(ptr) - 1
    y = np.zeros(n)
    for i in range(n):
        s = v[i]
        for p in range(ptr[i], diag[i]):
            s -= lu[p] * y[col[p]]
        y[i] = s
    z = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s = y[i]
        for p in range(diag[i] + 1, ptr[i + 1]):
            s -= lu[p] * z[col[p]]
        z[i] = s / lu[diag[i]]
    return z
