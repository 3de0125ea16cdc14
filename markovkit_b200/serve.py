"""Serving resolvent solves: a Python face of the request loop behind mk_server_*.

    srv = server(slots=4, precision="fp32")
    pid = srv.register(box, model)            # population_box / population_sector + reaction_diffusion
    t = srv.submit(pid, shift, b)             # b: host float64 array of the space's size
    x, result = srv.wait(t)
    srv.stats()                               # p50 / p99 latency, solves/s, resident bytes, ...

Each request is the reference's resolvent solve (shift I - Q) x = b with sector_multigrid and
GMRES at a relative true-residual target (tests/test_rdme.cpp:225-251), on a solver kept
resident on the device per (problem, shift); several requests run at once on separate streams.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as _L
from ._lib import MK_ENOTCONV, ServerOptions, ServerResult, ServerStats, check, load


@dataclass
class request_result:
    ticket: int
    status: int
    iterations: int
    residual: float
    latency_ms: float
    queue_ms: float
    solve_ms: float
    batched: int = 1


class server:
    def __init__(self, slots: int = 4, precision: str = "fp32", hbm_budget: int = 0, smoother: str = "jacobi",
                 restart: int = 30, max_iterations: int = 5000, rel_tolerance: float = 1e-10,
                 batch: int = 4, coarsest_size: int = 256):
        lib = load()
        o = ServerOptions()
        lib.mk_server_options_default(C.byref(o))
        o.slots = int(slots)
        o.hbm_budget = int(hbm_budget)
        o.precision = {"fp64": 0, "fp32": 1}[precision]
        o.smoother = {"auto": -1, "jacobi": 0, "gauss_seidel": 1, "ilu0": 2, "aggregate_block": 3}[smoother]
        o.restart = int(restart)
        o.max_iterations = int(max_iterations)
        o.rel_tolerance = float(rel_tolerance)
        o.batch = int(batch)
        o.coarsest_size = int(coarsest_size)
        self._h = C.c_void_p()
        check(lib.mk_server_create(C.byref(o), C.byref(self._h)))
        self._sizes = {}
        self._pending = {}  # ticket -> (b, x) kept alive until waited

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h and h.value and _L._lib is not None:
            _L._lib.mk_server_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def register(self, space, model) -> int:
        """copies a population space and a reaction_diffusion model into the server"""
        from .api import _Model

        m = _Model(model, tuple_max=list(space.limits))
        pid = C.c_int()
        check(load().mk_server_register(self._h, space._h, m._h, C.byref(pid)))
        self._sizes[pid.value] = space.size()
        return pid.value

    def footprint(self, problem: int) -> int:
        b = C.c_size_t()
        check(load().mk_server_footprint(self._h, int(problem), C.byref(b)))
        return b.value

    def submit(self, problem: int, shift: float, b: np.ndarray, x: np.ndarray | None = None) -> int:
        n = self._sizes[problem]
        b = np.ascontiguousarray(b, dtype=np.float64)
        if b.shape != (n,):
            raise ValueError(f"b must have {n} entries")
        if x is None:
            x = np.empty(n, dtype=np.float64)
        t = C.c_int64()
        check(load().mk_server_submit(self._h, int(problem), float(shift), C.c_void_p(b.ctypes.data),
                                      C.c_void_p(x.ctypes.data), C.byref(t)))
        self._pending[t.value] = (b, x)
        return t.value

    def wait(self, ticket: int, timeout_ms: float | None = None, allow: tuple = ()):
        """Block until the request is done (at most timeout_ms: MkError MK_ETIMEOUT, the request
        stays pending) and return (x, request_result). A request that ended with a status other
        than MK_OK or MK_ENOTCONV raises MkError, unless the status is in `allow`."""
        r = ServerResult()
        if timeout_ms is None:
            rc = load().mk_server_wait(self._h, int(ticket), C.byref(r))
        else:
            rc = load().mk_server_wait_for(self._h, int(ticket), float(timeout_ms), C.byref(r))
        check(rc, allow=(MK_ENOTCONV, *allow))
        b, x = self._pending.pop(ticket, (None, None))
        return x, request_result(r.ticket, r.status, r.iterations, r.residual, r.latency_ms, r.queue_ms, r.solve_ms,
                                 r.batched)

    def cancel(self, ticket: int) -> None:
        """Remove a request that no worker has taken yet; waiting on it then gives status
        MK_ECANCELED. MkError MK_EINVAL once it has started or finished."""
        check(load().mk_server_cancel(self._h, int(ticket)))

    def drain(self) -> None:
        check(load().mk_server_drain(self._h))

    def stats(self) -> dict:
        s = ServerStats()
        check(load().mk_server_stats_get(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}


def serving_problem(model: str, voxels: int, cap: int):
    """The population box and RDME model of a serving-workload request
    (markovkit_b200.inputs.serving_requests): unit diffusion; birth 0.05 vol and death 0.02 n
    for the birth-death boxes, annihilation A + B -> 0 at 10 nA nB / vol on the 2-D box {1, 1}.
    cfg0-2 use the unit domain (spacing 1 / cells). The 1-D boxes of 64-256 voxels keep
    configuration 0's voxel size 1/16 (a longer line): on the unit domain their jump rates reach
    8 D V^2 per state, and at small shifts the FP64 residual floor eps ||A|| / s lies above the
    1e-10 target (V = 208, cap 3, s = 0.113 stalls at 2.6e-10 relative in FP64 GMRES)."""
    from . import api as mk

    dim = {"cfg0": 1, "cfg1": 2, "cfg2": 3, "bd1d": 1}[model]
    cells = round(voxels ** (1.0 / dim))
    h = 1.0 / 16 if model == "bd1d" else 1.0 / cells
    if model == "cfg1":
        D, caps = [1.0, 1.0], [cap, cap]
        rx = [mk.local_reaction([-1, -1], lambda n, vol: 10.0 * n[0] * n[1] / vol)]
    else:
        D, caps = [1.0], [cap]
        rx = [mk.local_reaction([1], lambda n, vol: 0.05 * vol), mk.local_reaction([-1], lambda n, vol: 0.02 * n[0])]
    dom = mk.voxel_domain(mk.grid([cells] * dim, [h] * dim), D)
    assert cells ** dim == voxels
    return mk.population_box(voxels, caps), mk.reaction_diffusion(dom, rx)
