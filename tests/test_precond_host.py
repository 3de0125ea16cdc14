"""CPU checks of the preconditioner layer: the ILU(0) oracle (oracle/ilu0.py) against an exact
answer, and the C ABI's refusal of malformed matrices before any device work."""

import ctypes as C

import numpy as np
import pytest

from markovkit_b200 import _lib
from oracle.ilu0 import ilu0_factor, ilu0_solve


def _csr(dense):
    ptr, col, val = [0], [], []
    for row in dense:
        for j, a in enumerate(row):
            if a != 0.0:
                col.append(j)
                val.append(a)
        ptr.append(len(col))
    return np.array(ptr, dtype=np.int64), np.array(col, dtype=np.int64), np.array(val)


def test_oracle_ilu0_is_exact_on_a_tridiagonal_matrix():
    """ILU(0) of a tridiagonal matrix fills nothing, so it is the exact LU: z = A^-1 v"""
    rng = np.random.default_rng(3)
    n = 40
    A = np.diag(4.0 + rng.uniform(size=n)) + np.diag(-rng.uniform(size=n - 1), 1) + np.diag(-rng.uniform(size=n - 1), -1)
    ptr, col, val = _csr(A)
    lu, diag = ilu0_factor(ptr, col, val)
    v = rng.uniform(-1.0, 1.0, n)
    np.testing.assert_allclose(ilu0_solve(ptr, col, lu, diag, v), np.linalg.solve(A, v), rtol=1e-12, atol=1e-14)


def test_oracle_ilu0_drops_fill_outside_the_pattern():
    """on an arrow-shaped pattern the product L U matches A on A's pattern only"""
    A = np.array([[4.0, 1.0, 1.0], [1.0, 4.0, 0.0], [1.0, 0.0, 4.0]])
    ptr, col, val = _csr(A)
    lu, diag = ilu0_factor(ptr, col, val)
    L, U = np.eye(3), np.zeros((3, 3))
    for i in range(3):
        for p in range(ptr[i], ptr[i + 1]):
            (L if col[p] < i else U)[i, col[p]] = lu[p]
    prod = L @ U
    mask = A != 0.0
    np.testing.assert_allclose(prod[mask], A[mask], rtol=1e-14)
    assert prod[1, 2] != 0.0  # the dropped fill


def _create_ilu0(ptr, col, val):
    lib = _lib.load()
    out = C.c_void_p()
    I64P = C.POINTER(C.c_int64)
    rc = lib.mk_precond_create_ilu0(len(ptr) - 1, ptr.ctypes.data_as(I64P), col.ctypes.data_as(I64P),
                                    val.ctypes.data_as(C.POINTER(C.c_double)), None, C.byref(out))
    return rc, out


@pytest.mark.parametrize("case", ["no_diagonal", "unsorted", "out_of_range", "bad_ptr"])
def test_malformed_matrices_are_refused_on_the_host(case):
    ptr = np.array([0, 2, 4], dtype=np.int64)
    col = np.array([0, 1, 0, 1], dtype=np.int64)
    val = np.array([2.0, 1.0, 1.0, 2.0])
    if case == "no_diagonal":
        col = np.array([0, 1, 0, 0], dtype=np.int64)[[0, 1, 2]]
        ptr = np.array([0, 2, 3], dtype=np.int64)
        val = val[:3]
    elif case == "unsorted":
        col = np.array([1, 0, 0, 1], dtype=np.int64)
    elif case == "out_of_range":
        col = np.array([0, 2, 0, 1], dtype=np.int64)
    else:
        ptr = np.array([0, 3, 2], dtype=np.int64)
    rc, out = _create_ilu0(ptr, col, val)
    assert rc == _lib.MK_EINVAL and not out.value
    assert _lib.load().mk_last_error()


def test_null_callback_and_empty_diagonal_are_refused():
    lib = _lib.load()
    out = C.c_void_p()
    assert lib.mk_precond_create_host(4, _lib.PRECOND_HOST_FN(0), None, C.byref(out)) == _lib.MK_EINVAL
    d = np.ones(1)
    assert lib.mk_precond_create_diagonal(0, d.ctypes.data_as(C.POINTER(C.c_double)), C.byref(out)) == _lib.MK_EINVAL
