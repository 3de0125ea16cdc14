"""CPU checks of the SSA oracle (oracle/ssa_port.py) and of the SSA C ABI's argument checks.

The Philox4x32-10 restatement is pinned by the known-answer vectors its authors publish with
Random123 (kat_vectors: philox4x32 with 10 rounds); the Gillespie restatement by the reference
test's own cases (tests/test_ssa.cpp:23-63): the birth-death mean, the jump limit."""

import ctypes as C
import math

import numpy as np
import pytest

from markovkit_b200 import _lib
from oracle.ssa_port import Stream, gillespie, philox4x32_10


def test_philox_known_answers():
    assert philox4x32_10((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert philox4x32_10((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF)) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert philox4x32_10((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == (
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def test_uniforms_lie_in_unit_interval():
    s = Stream(123, 4)
    u = np.array([s.uniform() for _ in range(20000)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.01 and abs(u.var() - 1 / 12) < 0.005


def _birth_death_tables(birth, death, cap):
    n = np.arange(cap + 1, dtype=np.float64)
    return [[1], [-1]], [np.full(cap + 1, birth), death * n], [cap]


def test_oracle_birth_death_mean():
    """tests/test_ssa.cpp:23-36 with the oracle's stream: 2000 paths, mean within 0.5"""
    change, rates, bounds = _birth_death_tables(5.0, 0.1, 200)
    finals = [gillespie(change, rates, bounds, [0], 2.0, 100, p)[1][-1][0] for p in range(2000)]
    exact = (5.0 / 0.1) * (1.0 - math.exp(-0.1 * 2.0))
    assert abs(np.mean(finals) - exact) < 0.5


def test_oracle_jump_limit():
    """tests/test_ssa.cpp:52-57: five jumps give six states; a cut path ends at its last jump"""
    times, states = gillespie([[1]], [np.ones(101)], [100], [0], 100.0, 12345, 0, max_jumps=5)
    assert len(states) == 6 and times[-1] < 100.0


def test_ssa_arguments_checked_on_the_host():
    lib = _lib.load()
    q = _lib.SsaProblem()
    lib.mk_ssa_problem_default(C.byref(q))
    assert q.max_jumps == 2 ** 63 - 1 and q.paths == 1 and q.leap_epsilon == 0.03
    bounds = (C.c_int * 1)(10)
    initial = (C.c_int * 1)(11)  # outside the box
    q.n_species, q.n_reactions = 1, 0
    q.bounds, q.initial, q.final_time = bounds, initial, 1.0
    fin, st = (C.c_int * 1)(), (C.c_int * 1)()
    steps = (C.c_int64 * 1)()
    out = _lib.SsaOutput(fin, None, steps, st, None, None, None)
    assert lib.mk_ssa_run(C.byref(q), C.byref(out), None) == _lib.MK_EINVAL
    initial[0] = 3
    q.method = 7
    assert lib.mk_ssa_run(C.byref(q), C.byref(out), None) == _lib.MK_EINVAL
    q.method = 0
    obs = (C.c_double * 2)(0.5, 0.25)  # not sorted
    q.n_observations, q.observation_times = 2, obs
    assert lib.mk_ssa_run(C.byref(q), C.byref(out), None) == _lib.MK_EINVAL


@pytest.mark.parametrize("seed", [0, 2 ** 40 + 7])
def test_stream_depends_on_seed_and_path_only(seed):
    a = [Stream(seed, 3).uniform() for _ in range(3)]
    s = Stream(seed, 3)
    b = [s.uniform() for _ in range(3)]
    assert a[0] == b[0]
    assert Stream(seed, 4).uniform() != b[0]
