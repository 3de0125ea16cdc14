"""Python mirror of MarkovKit's Krylov and adaptive finite state projection over the C ABI.

Names and argument meaning follow markovkit/fsp.hpp and markovkit/reaction_network.hpp:
reaction_network{reactions: [reaction{change, rate}]}, krylov_fsp_options (fsp.hpp:190-202)
with inside = box(bounds) (fsp.hpp:26-35), solve_krylov_fsp(model, initial, final_time,
options) -> fsp_solution{times, snapshots} (fsp.hpp:86-107,207-254). The propensities are
tabulated here over the box and the whole attempt loop runs on the GPU, many instances per
launch (fsp_batch). The region is box(bounds), box(bound) or everywhere() (the default, None):
an everywhere() instance runs in a box whose bounds double (2b + 1) on each species an expansion
would have crossed and runs again until no expansion met the box (mk_fsp_result.clipped), so its
support grew exactly as an unbounded region lets it. Differences from the reference: krylov_dim
is at most 30, and only the initial and final distributions are saved (save_every has no
counterpart).
"""

from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib as _L
from ._lib import MK_ENOTCONV, FspOptions, FspProblem, FspResult, check, load


@dataclass
class reaction:
    """reaction_network::reaction (reaction_network.hpp:11-16): a change vector and a rate.

    rate(x) gets the states as an int array of shape (count, n_species) and returns their
    rates (shape (count,)); a rate written for one state (returning a scalar) also works.
    """

    change: Sequence[int]
    rate: Callable


@dataclass
class reaction_network:
    reactions: list = field(default_factory=list)


@dataclass
class box:
    """box(bounds): 0 <= x[s] <= bounds[s] (fsp.hpp:26-35); box(bound) with one int bounds every
    species by it (fsp.hpp:37-42) once the species count is known (resolved)."""

    bounds: Sequence[int]

    def resolved(self, species: int) -> "box":
        if isinstance(self.bounds, (int, np.integer)):
            return box([int(self.bounds)] * species)
        return self

    def size(self) -> int:
        return int(np.prod([b + 1 for b in self.bounds], dtype=np.int64))

    def states(self) -> np.ndarray:
        """every state of the box, in box order (species 0 most significant)"""
        axes = [np.arange(b + 1) for b in self.bounds]
        grids = np.meshgrid(*axes, indexing="ij")
        return np.stack([g.reshape(-1) for g in grids], axis=1).astype(np.int64)

    def index(self, x: Sequence[int]) -> int:
        i = 0
        for s, b in enumerate(self.bounds):
            i = i * (b + 1) + int(x[s])
        return i


@dataclass
class krylov_fsp_options:
    inside: Optional[box] = None
    tolerance: float = 1e-6
    initial_step: float = 1.0
    step_growth: float = 2.0
    drop_probability: float = 1e-10
    drop_derivative: float = 1e-16
    layers: int = 1
    max_steps: int = 1 << 28
    krylov_dim: int = 30
    krylov_tol: float = 1e-8

    def _c(self) -> FspOptions:
        o = FspOptions()
        load().mk_fsp_options_default(C.byref(o))
        o.tolerance = self.tolerance
        o.initial_step = self.initial_step
        o.step_growth = self.step_growth
        o.drop_probability = self.drop_probability
        o.drop_derivative = self.drop_derivative
        o.layers = self.layers
        o.krylov_dim = self.krylov_dim
        o.max_steps = self.max_steps
        o.krylov_tol = self.krylov_tol
        return o


@dataclass
class adaptive_fsp_options:
    """adaptive_fsp_options (fsp.hpp:108-121) with inside = box(bounds). sampled_expansion (and
    its seed) has no device counterpart: only the full ring expansion runs."""

    inside: Optional[box] = None
    step_scale: float = 1.0
    prune_fraction: float = 0.1
    flux_tolerance: float = 1e-6
    min_probability: float = 0.0
    layers: int = 1
    sampled_expansion: bool = False
    seed: int = 42
    save_every: int = 1000
    max_steps: int = 1 << 28
    krylov_dim: int = 30
    krylov_tol: float = 1e-8

    def _c(self) -> FspOptions:
        if self.sampled_expansion:
            raise ValueError("adaptive FSP on the device expands every neighbour (sampled_expansion = False)")
        o = FspOptions()
        load().mk_fsp_options_default(C.byref(o))
        o.method = 1
        o.step_scale = self.step_scale
        o.prune_fraction = self.prune_fraction
        o.flux_tolerance = self.flux_tolerance
        o.min_probability = self.min_probability
        o.layers = self.layers
        o.max_steps = self.max_steps
        o.krylov_dim = self.krylov_dim
        o.krylov_tol = self.krylov_tol
        return o


@dataclass
class distribution:
    """The supported states (rows, box order) and their probabilities (distribution.hpp)."""

    states: np.ndarray
    probabilities: np.ndarray

    def size(self) -> int:
        return len(self.probabilities)

    def means(self) -> np.ndarray:
        return (self.probabilities[:, None] * self.states).sum(axis=0)

    def as_dict(self) -> dict:
        return {tuple(int(v) for v in x): float(p) for x, p in zip(self.states, self.probabilities)}


@dataclass
class fsp_solution:
    times: list
    snapshots: list
    attempts: int = 0
    accepted: int = 0

    def means(self) -> np.ndarray:
        return np.stack([d.means() for d in self.snapshots])


def tabulate(model: reaction_network, region: box) -> tuple[np.ndarray, np.ndarray]:
    """change (R x S) and rates (R x box size) of the network over the box."""
    states = region.states()
    S = states.shape[1]
    R = len(model.reactions)
    change = np.zeros((R, S), dtype=np.int32)
    rates = np.zeros((R, len(states)), dtype=np.float64)
    for r, rx in enumerate(model.reactions):
        ch = np.asarray(rx.change, dtype=np.int32)
        if ch.shape != (S,):
            raise ValueError("change vector length differs from the number of species")
        change[r] = ch
        vals = None
        try:
            out = np.asarray(rx.rate(states), dtype=np.float64)
            if out.shape == (len(states),):
                vals = out
        except Exception:
            vals = None
        if vals is None:
            vals = np.array([float(rx.rate(tuple(int(v) for v in x))) for x in states])
        rates[r] = vals
    return change, rates


class everywhere:
    """everywhere() (fsp.hpp:20-24): the region of every state; the device runs it in a box that
    grows until no expansion meets it. options.inside = None means the same."""


def _first_box(initial) -> box:
    return box([max(2 * int(v), int(v) + 16) for v in initial])


_LARGEST_AUTO_BOX = 1 << 26


class _Problem:
    """one instance, with the arrays its mk_fsp_problem points at kept alive"""

    def __init__(self, model, initial, final_time, options):
        if not isinstance(options.inside, box):
            raise ValueError("an fsp_batch instance needs a box region (options.inside = box(bounds)); "
                             "solve_krylov_fsp and solve_adaptive_fsp also take everywhere()")
        options = dataclasses.replace(options, inside=options.inside.resolved(len(initial)))
        self.region = options.inside
        self.bounds = np.ascontiguousarray(options.inside.bounds, dtype=np.int32)
        self.change, self.rates = tabulate(model, options.inside)
        self.change = np.ascontiguousarray(self.change)
        self.rates = np.ascontiguousarray(self.rates)
        self.initial = np.ascontiguousarray(initial, dtype=np.int32)
        self.c = FspProblem()
        self.c.n_species = len(self.bounds)
        self.c.n_reactions = self.change.shape[0]
        self.c.bounds = self.bounds.ctypes.data_as(C.POINTER(C.c_int))
        self.c.change = self.change.ctypes.data_as(C.POINTER(C.c_int))
        self.c.rates = self.rates.ctypes.data_as(C.POINTER(C.c_double))
        self.c.initial = self.initial.ctypes.data_as(C.POINTER(C.c_int))
        self.c.final_time = float(final_time)
        self.c.options = options._c()

    def rate_bytes(self) -> int:
        return self.rates.nbytes


def _stream(stream=None) -> C.c_void_p:
    if stream is None:
        import torch

        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class fsp_batch:
    """Many solve_krylov_fsp runs resident on the device, run by one persistent kernel."""

    def __init__(self, problems):
        self._h = C.c_void_p()
        self.problems = [p if isinstance(p, _Problem) else _Problem(*p) for p in problems]
        arr = (FspProblem * len(self.problems))(*[p.c for p in self.problems])
        lib = load()
        check(lib.mk_fsp_batch_create(len(self.problems), arr, C.byref(self._h)))
        total = C.c_int64()
        offsets = (C.c_int64 * len(self.problems))()
        check(lib.mk_fsp_batch_output_size(self._h, C.byref(total), offsets))
        self.total = total.value
        self.offsets = np.array(offsets[:], dtype=np.int64)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _L._lib is not None:
            _L._lib.mk_fsp_batch_destroy(h)
            self._h = C.c_void_p()

    def __len__(self) -> int:
        return len(self.problems)

    def set_shape(self, threads: int, blocks: int = 0) -> None:
        check(load().mk_fsp_batch_set_shape(self._h, int(threads), int(blocks)))

    def shape(self) -> tuple[int, int]:
        t, b = C.c_int(), C.c_int()
        check(load().mk_fsp_batch_get_shape(self._h, C.byref(t), C.byref(b)))
        return t.value, b.value

    def autotune(self, sample: int = 0, stream=None) -> tuple[int, int]:
        check(load().mk_fsp_batch_autotune(self._h, int(sample), _stream(stream)))
        return self.shape()

    def run(self, stream=None) -> None:
        check(load().mk_fsp_batch_run(self._h, _stream(stream)))

    def device_output_ptr(self) -> int:
        p = C.c_void_p()
        check(load().mk_fsp_batch_device_output(self._h, C.byref(p)))
        return p.value

    def results(self, stream=None, with_output: bool = True):
        """(dense output over all boxes or None, list of FspResult); raises on a failed instance
        other than stopping early (MK_ENOTCONV, reported per result)"""
        out = np.empty(self.total, dtype=np.float64) if with_output else None
        res = (FspResult * len(self.problems))()
        optr = out.ctypes.data_as(C.POINTER(C.c_double)) if with_output else None
        check(load().mk_fsp_batch_results(self._h, optr, res, _stream(stream)), allow=(MK_ENOTCONV,))
        return out, list(res)

    def solutions(self, stream=None) -> list:
        out, res = self.results(stream)
        sols = []
        for k, (p, r) in enumerate(zip(self.problems, res)):
            dense = out[self.offsets[k] : self.offsets[k] + p.region.size()]
            nz = np.nonzero(dense)[0]
            states = p.region.states()[nz]
            x0 = distribution(p.initial[None, :].astype(np.int64), np.ones(1))
            sols.append(
                fsp_solution(
                    times=[0.0, r.time],
                    snapshots=[x0, distribution(states, dense[nz].copy())],
                    attempts=r.attempts,
                    accepted=r.accepted,
                )
            )
        return sols


def _solve(problems, stream=None, autotune: bool = False) -> list:
    """every (model, initial, final_time, options) in one launch; everywhere() instances run
    again in grown boxes until no expansion met their box"""
    problems = [tuple(p) for p in problems]
    automatic = [not isinstance(p[3].inside, box) for p in problems]
    for p, auto in zip(problems, automatic):
        if auto and p[3].inside is not None and not isinstance(p[3].inside, everywhere):
            raise ValueError("the device FSP takes box(...) or everywhere() as the region")
    regions = [_first_box(p[1]) if auto else p[3].inside for p, auto in zip(problems, automatic)]
    sols: list = [None] * len(problems)
    pending = list(range(len(problems)))
    while pending:
        b = fsp_batch([(problems[k][0], problems[k][1], problems[k][2],
                        dataclasses.replace(problems[k][3], inside=regions[k])) for k in pending])
        if autotune:
            b.autotune(stream=stream)
        b.run(stream)
        _, res = b.results(stream, with_output=False)
        grown = []
        for q, k in enumerate(pending):
            if automatic[k] and res[q].clipped:
                bounds = [2 * v + 1 if res[q].clipped >> s & 1 else v for s, v in enumerate(regions[k].bounds)]
                regions[k] = box(bounds)
                if regions[k].size() > _LARGEST_AUTO_BOX:
                    raise ValueError("fsp: the everywhere() support outgrew a box of 2^26 states")
                grown.append(k)
        done = b.solutions(stream)
        for q, k in enumerate(pending):
            if k not in grown:
                sols[k] = done[q]
        pending = grown
    return sols


def solve_krylov_fsp(model: reaction_network, initial: Sequence[int], final_time: float,
                     options: Optional[krylov_fsp_options] = None, stream=None) -> fsp_solution:
    """solve_krylov_fsp (fsp.hpp:207-254) on the GPU."""
    return _solve([(model, initial, final_time, options or krylov_fsp_options())], stream)[0]


def solve_krylov_fsp_batch(problems, stream=None, autotune: bool = False) -> list:
    """solve_krylov_fsp for each (model, initial, final_time, options), in one launch."""
    return _solve(problems, stream, autotune)


def solve_adaptive_fsp(model: reaction_network, initial: Sequence[int], final_time: float,
                       options: Optional[adaptive_fsp_options] = None, stream=None) -> fsp_solution:
    """solve_adaptive_fsp (fsp.hpp:123-188) on the GPU: flux-controlled steps of expand,
    expv on the reflecting generator of the support, prune and renormalise."""
    return _solve([(model, initial, final_time, options or adaptive_fsp_options())], stream)[0]
