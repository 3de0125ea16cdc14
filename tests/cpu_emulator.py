"""Builds and binds tests/cpu/emulate.cpp: the product's shared row logic run on the CPU."""

from __future__ import annotations

import ctypes as C
import subprocess
from functools import lru_cache
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpu" / "emulate.cpp"
CSRC = ROOT / "markovkit_b200" / "csrc"
OUT = ROOT / "tests" / "cpu" / "_build" / "libemulate.so"


@lru_cache(maxsize=1)
def lib() -> C.CDLL:
    deps = [SRC, *CSRC.glob("*.cuh"), CSRC / "host_model.hpp"]
    if not OUT.exists() or any(d.stat().st_mtime > OUT.stat().st_mtime for d in deps):
        OUT.parent.mkdir(parents=True, exist_ok=True)
        subprocess.run(
            ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-I", str(CSRC), str(SRC), "-o", str(OUT)],
            check=True,
        )
    return C.CDLL(str(OUT))


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def rate_table(reactions, tmax, volume):
    """Tabulate rate(counts, volume) over all count tuples 0..tmax (species 0 most significant)."""
    shape = [t + 1 for t in tmax]
    out = np.zeros((len(reactions), int(np.prod(shape))))
    for r, (_, fn) in enumerate(reactions):
        for k, counts in enumerate(np.ndindex(*shape)):
            out[r, k] = fn(list(counts), volume)
    return out


def generator(dim, dims, spacing, D, reactions, limits, is_box=True, absorbing=True, shift=0.0, x=None, csr=False):
    L = lib()
    S = len(D)
    dims_a = np.array(list(dims) + [1] * (3 - dim), dtype=np.int64)
    sp_a = np.array(list(spacing) + [1.0] * (3 - dim), dtype=np.float64)
    D_a = np.array(D, dtype=np.float64)
    lim = np.array(limits, dtype=np.int32)
    R = len(reactions)
    change = np.array([c for ch, _ in reactions for c in ch] or [0], dtype=np.int32)
    tmax = np.array(limits, dtype=np.int32)
    vol = float(np.prod(spacing))
    rates = rate_table(reactions, list(limits), vol).ravel() if R else np.zeros(1)
    err = C.create_string_buffer(256)
    fn = L.emu_generator
    fn.restype = C.c_int64
    args = [C.c_int(dim), _d(dims_a), _d(sp_a), C.c_int(S), _d(D_a), C.c_int(R), _d(change), _d(tmax), _d(rates), C.c_int(int(is_box)), _d(lim), C.c_int(int(absorbing)), C.c_double(shift)]
    n = fn(*args, None, None, None, None, None, err, C.c_int(int(csr)))
    if n < 0:
        raise ValueError(err.value.decode())
    if x is None:
        x = np.zeros(n)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = {k: np.zeros(n) for k in ("exit", "leak", "Qx", "Ax")}
    n = fn(*args, _d(x), _d(out["exit"]), _d(out["leak"]), _d(out["Qx"]), _d(out["Ax"]), err, C.c_int(int(csr)))
    if n < 0:
        raise ValueError(err.value.decode())
    return out


def matrix(dim, dims, spacing, D, reactions, limits, is_box=True, absorbing=True, shift=0.0, sign=1.0, csr=False):
    """sign * (Q - shift I) assembled from the row visits (scipy CSR, equal positions summed)."""
    import scipy.sparse as sp

    L = lib()
    S = len(D)
    dims_a = np.array(list(dims) + [1] * (3 - dim), dtype=np.int64)
    sp_a = np.array(list(spacing) + [1.0] * (3 - dim), dtype=np.float64)
    D_a = np.array(D, dtype=np.float64)
    lim = np.array(limits, dtype=np.int32)
    R = len(reactions)
    change = np.array([c for ch, _ in reactions for c in ch] or [0], dtype=np.int32)
    tmax = np.array(limits, dtype=np.int32)
    vol = float(np.prod(spacing))
    rates = rate_table(reactions, list(limits), vol).ravel() if R else np.zeros(1)
    err = C.create_string_buffer(256)
    fn = L.emu_matrix
    fn.restype = C.c_int64
    args = [C.c_int(dim), _d(dims_a), _d(sp_a), C.c_int(S), _d(D_a), C.c_int(R), _d(change), _d(tmax),
            _d(rates), C.c_int(int(is_box)), _d(lim), C.c_int(int(absorbing)), C.c_double(shift), C.c_double(sign)]
    n = fn(*args, None, None, None, C.c_int64(0), err, C.c_int(int(csr)))
    if n < 0:
        raise ValueError(err.value.decode())
    row = np.zeros(n, dtype=np.int64)
    col = np.zeros(n, dtype=np.int64)
    val = np.zeros(n)
    N = int(emu_size(dim, dims, spacing, D, reactions, limits, is_box, absorbing, csr))
    m = fn(*args, _d(row), _d(col), _d(val), C.c_int64(n), err, C.c_int(int(csr)))
    if m != n:
        raise ValueError(err.value.decode() or "triplet count changed")
    out = sp.coo_matrix((val, (row, col)), shape=(N, N)).tocsr()
    out.sum_duplicates()
    out.sort_indices()
    return out


def emu_size(dim, dims, spacing, D, reactions, limits, is_box=True, absorbing=True, csr=False):
    return len(generator(dim, dims, spacing, D, reactions, limits, is_box, absorbing, csr=csr)["exit"])


def states(V, limits, is_box=True):
    L = lib()
    S = len(limits)
    lim = np.array(limits, dtype=np.int32)
    err = C.create_string_buffer(256)
    fn = L.emu_states
    fn.restype = C.c_int64
    n = fn(C.c_int(V), C.c_int(S), _d(lim), C.c_int(int(is_box)), None, None, err)
    if n < 0:
        raise ValueError(err.value.decode())
    st = np.zeros((n, V * S), dtype=np.int32)
    rk = np.zeros(n, dtype=np.int64)
    fn(C.c_int(V), C.c_int(S), _d(lim), C.c_int(int(is_box)), _d(st), _d(rk), err)
    return st, rk


def transfer(dim, dims, spacing, totals, c, g):
    L = lib()
    S = len(totals)
    dims_a = np.array(list(dims) + [1] * (3 - dim), dtype=np.int64)
    sp_a = np.array(list(spacing) + [1.0] * (3 - dim), dtype=np.float64)
    tot = np.array(totals, dtype=np.int32)
    err = C.create_string_buffer(256)
    nc = C.c_int64()
    fn = L.emu_transfer
    fn.restype = C.c_int64
    nf = fn(C.c_int(dim), _d(dims_a), _d(sp_a), C.c_int(S), _d(tot), None, None, None, None, C.byref(nc), err)
    if nf < 0:
        raise ValueError(err.value.decode())
    c = np.ascontiguousarray(c, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    Pc = np.zeros(nf)
    Rg = np.zeros(nc.value)
    r = fn(C.c_int(dim), _d(dims_a), _d(sp_a), C.c_int(S), _d(tot), _d(c), _d(g), _d(Pc), _d(Rg), C.byref(nc), err)
    if r < 0:
        raise ValueError(err.value.decode())
    return Pc, Rg


def stencil_check(dim, dims, spacing, D, reactions, limits, is_box=True, absorbing=True):
    """Rows compared by emu_stencil_check (stencil forms == general visit, bit for bit)."""
    L = lib()
    S = len(D)
    dims_a = np.array(list(dims) + [1] * (3 - dim), dtype=np.int64)
    sp_a = np.array(list(spacing) + [1.0] * (3 - dim), dtype=np.float64)
    D_a = np.array(D, dtype=np.float64)
    lim = np.array(limits, dtype=np.int32)
    R = len(reactions)
    change = np.array([c for ch, _ in reactions for c in ch] or [0], dtype=np.int32)
    tmax = np.array(limits, dtype=np.int32)
    vol = float(np.prod(spacing))
    rates = rate_table(reactions, list(limits), vol).ravel() if R else np.zeros(1)
    err = C.create_string_buffer(256)
    fn = L.emu_stencil_check
    fn.restype = C.c_int64
    n = fn(C.c_int(dim), _d(dims_a), _d(sp_a), C.c_int(S), _d(D_a), C.c_int(R), _d(change), _d(tmax), _d(rates),
           C.c_int(int(is_box)), _d(lim), C.c_int(int(absorbing)), err)
    if n < 0:
        raise ValueError(err.value.decode())
    return int(n)
