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


def fsp_batch_instances(seed: int = 3, count: int = 512, final_time: float = 2.0,
                        tolerance: float = 1e-8) -> list:
    """Seeded Krylov-FSP instances of the batching workload: the first half birth-death
    ({+1} at b, {-1} at d x; b ~ U(1, 20), d ~ U(0.05, 0.5), box bound ~ U{99..1999}, so 100 to
    2000 states), the second half toggle switches ({+1,0} at a1 / (1 + y^n1), {0,+1} at
    a2 / (1 + x^n2), unit degradation; a ~ U(20, 60), n ~ U(1.5, 3), bounds ~ U{50..300}).
    Instance k draws u(seed, 8k + j), j < 6. All start from the delta at 0."""
    u = uniform01(seed, 8 * count)
    out = []
    for k in range(count):
        v = u[8 * k : 8 * k + 8]
        if k < count // 2:
            out.append({
                "family": "birth_death",
                "birth": 1.0 + 19.0 * v[0],
                "death": 0.05 + 0.45 * v[1],
                "bounds": [99 + int(1901 * v[2])],
                "initial": [0],
                "final_time": final_time,
                "tolerance": tolerance,
            })
        else:
            out.append({
                "family": "toggle",
                "a1": 20.0 + 40.0 * v[0],
                "a2": 20.0 + 40.0 * v[1],
                "n1": 1.5 + 1.5 * v[2],
                "n2": 1.5 + 1.5 * v[3],
                "bounds": [50 + int(251 * v[4]), 50 + int(251 * v[5])],
                "initial": [0, 0],
                "final_time": final_time,
                "tolerance": tolerance,
            })
    return out


def fsp_instance_line(inst: dict, krylov_tol: float = 1e-8, krylov_dim: int = 30,
                      max_steps: int | None = None) -> str:
    """One instance in the line format of the oracle's Krylov-FSP driver (max_steps: the
    attempt cap of krylov_fsp_options, default the reference's)."""
    g = lambda x: repr(float(x))  # noqa: E731 - shortest round-trip decimal
    tail = [] if max_steps is None else [f"max_steps={int(max_steps)}"]
    if inst["family"] == "birth_death":
        return " ".join(["birth_death", g(inst["birth"]), g(inst["death"]), str(inst["bounds"][0]),
                         g(inst["final_time"]), g(inst["tolerance"]), g(krylov_tol), str(krylov_dim),
                         str(inst["initial"][0]), *tail])
    return " ".join(["toggle", g(inst["a1"]), g(inst["a2"]), g(inst["n1"]), g(inst["n2"]),
                     str(inst["bounds"][0]), str(inst["bounds"][1]), g(inst["final_time"]),
                     g(inst["tolerance"]), g(krylov_tol), str(krylov_dim), str(inst["initial"][0]),
                     str(inst["initial"][1]), *tail])


SERVING_MODELS = ("cfg0", "cfg1", "cfg2", "bd1d")


def serving_requests(seed: int = 4, count: int = 24, rate: float = 20.0) -> list:
    """Seeded resolvent requests of the serving workload, in arrival order: Poisson arrivals at
    `rate` per second; the model uniform over the 1-D 16-voxel birth-death box of cap 3 (cfg0),
    the 2-D 32 x 32 annihilation box {1, 1} (cfg1), the 3-D 16^3 birth-death box of cap 2 (cfg2)
    and a 1-D birth-death box of V voxels, V uniform over the multiples of 16 in [64, 256], and
    cap ~ U{2..4} (bd1d, 2,145 to 186,043,585 states); shift log-uniform in [0.1, 10];
    right-hand side Dirichlet(1) of seed rhs_seed. Request k draws u(seed, 8k + j), j < 5.
    V is a multiple of 16 because sector_multigrid halves the grid only while its length is
    even (markovkit/rdme/multigrid.hpp:24-42) and factors what is left densely: a 1-D grid that
    stops above 16 voxels leaves sectors of hundreds of thousands of states at cap 4."""
    u = uniform01(seed, 8 * count)
    fixed = {"cfg0": (16, 3), "cfg1": (1024, 1), "cfg2": (4096, 2)}
    out, t = [], 0.0
    for k in range(count):
        v = u[8 * k : 8 * k + 8]
        t += -float(np.log1p(-v[0])) / rate
        model = SERVING_MODELS[min(3, int(4 * v[1]))]
        voxels, cap = fixed.get(model, (64 + 16 * int(13 * v[2]), 2 + int(3 * v[3])))
        out.append({
            "arrival_s": t,
            "model": model,
            "voxels": voxels,
            "cap": cap,
            "shift": float(10.0 ** (-1.0 + 2.0 * v[4])),
            "rhs_seed": 1000 * seed + k,
        })
    return out
