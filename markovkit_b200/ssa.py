"""Stochastic simulation on the device: MarkovKit's gillespie and tau_leaping
(markovkit/ssa.hpp:42-113) for a reaction_network, many independent paths per launch
(mk_ssa_run, one path per thread).

The propensities are tabulated over a box, as for the device FSP; with no bounds given the box
starts around the initial state and doubles whenever a path would leave it. Path i is a function
of (seed, i) alone (Philox4x32-10), so a rerun on a wider box replays every path exactly. The
reference draws from a host generator: paths agree with it in distribution, not sample by sample.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import SsaOutput, SsaProblem, check, load
from .fsp import box, reaction_network, tabulate

_MAX_BOX = 1 << 26  # tabulated states, at most


@dataclass
class trajectory:
    """A piecewise-constant path: the chain is in states[k] from times[k] until times[k + 1]
    (ssa.hpp:14-39)."""

    times: list
    states: list

    def component(self, species: int) -> np.ndarray:
        return np.array([float(x[species]) for x in self.states])

    def indices_at(self, observation_times: Sequence[float]) -> list:
        out, k = [], 0
        for t in observation_times:
            while k + 1 < len(self.times) and self.times[k + 1] <= t:
                k += 1
            out.append(k)
        return out


@dataclass
class leap_options:
    """ssa.hpp:77-81: a fixed leap, or one from epsilon (expected jumps per leap)"""

    step: float = 0.0
    epsilon: float = 0.03
    min_step: float = 1e-6


@dataclass
class ssa_ensemble:
    """paths of one simulation: final states (paths x S), states at the observation times
    (paths x n_obs x S), jumps or leaps per path, statuses, and the box used"""

    final: np.ndarray
    observed: Optional[np.ndarray]
    steps: np.ndarray
    status: np.ndarray
    observation_times: np.ndarray
    bounds: list
    record_times: Optional[np.ndarray] = None
    record_states: Optional[np.ndarray] = None
    record_count: Optional[np.ndarray] = None

    def means(self) -> np.ndarray:
        """mean state at each observation time (n_obs x S)"""
        return self.observed.mean(axis=0)

    def final_means(self) -> np.ndarray:
        return self.final.mean(axis=0)

    def trajectory(self, path: int) -> trajectory:
        n = int(self.record_count[path])
        if n > self.record_times.shape[1]:
            raise ValueError("the trajectory was longer than the record kept")
        return trajectory([float(t) for t in self.record_times[path, :n]],
                          [[int(v) for v in x] for x in self.record_states[path, :n]])


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None and a.size else None


def _run(model: reaction_network, initial, final_time, paths, seed, method, max_jumps, leap, obs, bounds, record):
    initial = np.asarray(initial, dtype=np.int32)
    S = initial.size
    region = box([int(b) for b in bounds])
    change, rates = tabulate(model, region)
    change = np.ascontiguousarray(change, dtype=np.int32)
    rates = np.ascontiguousarray(rates, dtype=np.float64)
    bnd = np.asarray(bounds, dtype=np.int32)
    obs = np.ascontiguousarray(obs, dtype=np.float64)
    q = SsaProblem()
    load().mk_ssa_problem_default(C.byref(q))
    q.n_species, q.n_reactions = S, change.shape[0]
    q.bounds, q.change, q.rates, q.initial = _ptr(bnd, C.c_int), _ptr(change, C.c_int), _ptr(rates, C.c_double), _ptr(initial, C.c_int)
    q.final_time = float(final_time)
    q.method = method
    if max_jumps is not None:
        q.max_jumps = int(max_jumps)
    q.leap_step, q.leap_epsilon, q.leap_min_step = float(leap.step), float(leap.epsilon), float(leap.min_step)
    q.paths, q.seed = int(paths), int(seed) & 0xFFFFFFFFFFFFFFFF
    q.n_observations = obs.size
    q.observation_times = _ptr(obs, C.c_double)
    q.record = int(record)
    final = np.zeros((paths, S), dtype=np.int32)
    observed = np.zeros((paths, obs.size, S), dtype=np.int32) if obs.size else None
    steps = np.zeros(paths, dtype=np.int64)
    status = np.zeros(paths, dtype=np.int32)
    rt = np.zeros((paths, record)) if record else None
    rs = np.zeros((paths, record, S), dtype=np.int32) if record else None
    rn = np.zeros(paths, dtype=np.int32) if record else None
    out = SsaOutput(_ptr(final, C.c_int), _ptr(observed, C.c_int), _ptr(steps, C.c_int64), _ptr(status, C.c_int),
                    _ptr(rt, C.c_double), _ptr(rs, C.c_int), _ptr(rn, C.c_int))
    rc = load().mk_ssa_run(C.byref(q), C.byref(out), None)
    check(rc, allow=(_lib.MK_EOVERFLOW, _lib.MK_ENOTCONV))
    return rc, ssa_ensemble(final, observed, steps, status, obs, [int(b) for b in bounds], rt, rs, rn)


def simulate(model: reaction_network, initial: Sequence[int], final_time: float, paths: int, seed: int = 0,
             method: str = "gillespie", max_jumps: Optional[int] = None, leap: Optional[leap_options] = None,
             observation_times: Sequence[float] = (), bounds: Optional[Sequence[int]] = None,
             record: int = 0) -> ssa_ensemble:
    """`paths` independent paths from `initial` to final_time by Gillespie's direct method
    ("gillespie") or Poisson tau-leaping ("tau_leaping"), in one launch. With bounds None the
    propensity box grows until no path leaves it; with bounds given a path that would leave
    the box stops there with status MK_EOVERFLOW."""
    kind = {"gillespie": 0, "tau_leaping": 1}[method]
    leap = leap or leap_options()
    x0 = [int(v) for v in initial]
    grow = bounds is None
    b = [max(2 * v, v + 64) for v in x0] if grow else [int(v) for v in bounds]
    while True:
        rc, ens = _run(model, x0, final_time, paths, seed, kind, max_jumps, leap, observation_times, b, record)
        if rc != _lib.MK_EOVERFLOW or not grow:
            break
        size = int(np.prod([v + 1 for v in b], dtype=np.int64))
        if size * 2 ** len(b) > _MAX_BOX:
            raise OverflowError("ssa: the paths leave every propensity box of at most 2^26 states")
        b = [2 * v + 1 for v in b]
    if rc == _lib.MK_ENOTCONV:
        raise _lib.MkError(rc, load().mk_last_error().decode(errors="replace"))
    return ens


def _single(model, x, final_time, seed, method, max_jumps, leap):
    record = 1024
    while True:
        ens = simulate(model, x, final_time, 1, seed, method, max_jumps, leap, (), None, record)
        n = int(ens.record_count[0])
        if n <= record:
            return ens.trajectory(0)
        record = n


def gillespie(model: reaction_network, x: Sequence[int], final_time: float, seed: int = 0,
              max_jumps: Optional[int] = None) -> trajectory:
    """gillespie(model, x, final_time, random, max_jumps) (ssa.hpp:42-74): one path; `seed`
    stands in for the random generator"""
    return _single(model, x, final_time, seed, "gillespie", max_jumps, None)


def tau_leaping(model: reaction_network, x: Sequence[int], final_time: float, seed: int = 0,
                options: Optional[leap_options] = None) -> trajectory:
    """tau_leaping(model, x, final_time, random, leap_options) (ssa.hpp:83-111): one path"""
    return _single(model, x, final_time, seed, "tau_leaping", None, options)
