"""Seeded inputs, identical on the CPU oracle and GPU sides.

u(seed, i) = top 53 bits of splitmix64(splitmix64(seed) ^ i) / 2^53 — the same counter-based
generator as oracle/seeded.hpp. Uniform right-hand sides are u / sum(u) (sequential sum);
Dirichlet(1) ones are -log1p(-u) normalised the same way.
"""

from __future__ import annotations

import numpy as np

_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(z: np.ndarray) -> np.ndarray:
    z = (z + np.uint64(0x9E3779B97F4A7C15)) & _M
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M
    return z ^ (z >> np.uint64(31))


def uniform01(seed: int, n: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        s = _splitmix64(np.array([seed], dtype=np.uint64))[0]
        z = _splitmix64(np.arange(n, dtype=np.uint64) ^ s)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _sequential_normalise(v: np.ndarray) -> np.ndarray:
    total = float(np.add.accumulate(v)[-1]) if v.size else 1.0
    return v / total


def uniform_rhs(seed: int, n: int) -> np.ndarray:
    return _sequential_normalise(uniform01(seed, n))


def dirichlet_rhs(seed: int, n: int) -> np.ndarray:
    return _sequential_normalise(-np.log1p(-uniform01(seed, n)))
