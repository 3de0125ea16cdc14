"""Batched SSA on the GPU (markovkit/ssa.hpp:42-113 through mk_ssa_run).

- Sample by sample: device Gillespie paths equal the CPU restatement of oracle/ssa_port.py on the
  same Philox stream (states exact, jump times within 1e-12 relative: the two sides' log differ
  in the last place at most).
- The reference test's checks (tests/test_ssa.cpp:15-63): transitions with nonpositive rates or
  negative results are skipped, the Gillespie and tau-leaping birth-death means, the jump limit.
- In distribution: the final-time law of a birth-death process against its Poisson law, and a
  toggle switch's mean against the device Krylov FSP (5 standard errors).
"""

import math

import numpy as np
import pytest

from markovkit_b200 import _lib
from markovkit_b200.fsp import box, krylov_fsp_options, reaction, reaction_network, solve_krylov_fsp, tabulate
from markovkit_b200.fsp_models import birth_death, toggle
from markovkit_b200.ssa import gillespie, leap_options, simulate, tau_leaping
from oracle.ssa_port import gillespie as oracle_gillespie

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("family", ["birth_death", "toggle"])
def test_paths_match_oracle_sample_by_sample(cuda, family):
    if family == "birth_death":
        model, x0, bounds, T = birth_death(5.0, 0.1), [0], [200], 2.0
    else:
        model, x0, bounds, T = toggle(30.0, 25.0, 2.0, 2.5), [0, 0], [120, 120], 1.0
    change, rates = tabulate(model, box(bounds))
    ens = simulate(model, x0, T, 6, seed=100, bounds=bounds, record=4096)
    for p in range(6):
        times, states = oracle_gillespie(change.tolist(), rates, bounds, x0, T, 100, p)
        got = ens.trajectory(p)
        assert [tuple(s) for s in got.states] == states, (family, p)
        np.testing.assert_allclose(got.times, times, rtol=1e-12, atol=0.0)
        assert int(ens.steps[p]) == len(states) - 2


def test_transitions_skip_nonpositive_rates_and_negative_counts(cuda):
    """tests/test_ssa.cpp:15-21: from {3} only the birth is listed"""
    model = reaction_network([reaction([1], lambda x: np.full(len(x), 2.0)),
                              reaction([-1], lambda x: np.full(len(x), -1.0)),
                              reaction([-4], lambda x: np.full(len(x), 1.0))])
    jumped = 0
    for seed in range(20):
        path = gillespie(model, [3], 2.0, seed=seed)
        counts = [s[0] for s in path.states]
        if len(counts) > 2:  # at least one jump before the final time
            # from 3 the only listed jump is the birth; from 4 on the {-4} reaction is listed too
            assert counts[1] == 4
            jumped += 1
        assert all(b - a in (0, 1, -4) for a, b in zip(counts, counts[1:]))
    assert jumped >= 15


def test_reference_birth_death_means(cuda):
    """tests/test_ssa.cpp:23-49: Gillespie (2000 paths) within 0.5, tau-leaping (500) within 1.0"""
    model = birth_death(5.0, 0.1)
    exact = (5.0 / 0.1) * (1.0 - math.exp(-0.1 * 2.0))
    g = simulate(model, [0], 2.0, 2000, seed=100)
    assert abs(g.final_means()[0] - exact) < 0.5
    t = simulate(model, [0], 2.0, 500, seed=7, method="tau_leaping")
    assert abs(t.final_means()[0] - exact) < 1.0


def test_jump_limit(cuda):
    """tests/test_ssa.cpp:52-57: five jumps give six states; the path ends at its last jump"""
    model = reaction_network([reaction([1], lambda x: np.full(len(x), 1.0))])
    path = gillespie(model, [0], 100.0, seed=12345, max_jumps=5)
    assert len(path.states) == 6 and path.times[-1] < 100.0


def test_final_law_is_poisson(cuda):
    """from 0, birth b and death d x: Poisson with mean (b/d)(1 - e^{-d t}); 200,000 paths"""
    b, d, T, paths = 8.0, 0.5, 1.5, 200_000
    ens = simulate(birth_death(b, d), [0], T, paths, seed=3)
    lam = b / d * (1.0 - math.exp(-d * T))
    n = np.arange(40)
    pmf = np.exp(n * math.log(lam) - lam - np.array([math.lgamma(k + 1.0) for k in n]))
    emp = np.bincount(ens.final[:, 0], minlength=40)[:40] / paths
    se = np.sqrt(pmf * (1 - pmf) / paths)
    assert np.all(np.abs(emp - pmf) <= 5 * se + 1e-12)


def test_toggle_mean_matches_fsp(cuda):
    model = toggle(30.0, 25.0, 2.0, 2.5)
    T, paths = 1.0, 100_000
    ens = simulate(model, [0, 0], T, paths, seed=11, observation_times=[0.25, 0.5, 1.0])
    fsp = solve_krylov_fsp(model, [0, 0], T, krylov_fsp_options(inside=box([120, 120]), tolerance=1e-8))
    m_fsp = fsp.means()[-1]
    m_ssa = ens.means()[-1]
    se = ens.observed[:, -1, :].std(axis=0) / math.sqrt(paths)
    assert np.all(np.abs(m_ssa - m_fsp) <= 5 * se), (m_ssa, m_fsp, se)
    # the last observation time is final_time: the final state
    assert np.array_equal(ens.observed[:, -1, :], ens.final)


def test_observations_are_trajectory_states(cuda):
    model = toggle(30.0, 25.0, 2.0, 2.5)
    obs = [0.0, 0.1, 0.37, 0.8]
    ens = simulate(model, [0, 0], 1.0, 16, seed=5, observation_times=obs, record=4096)
    for p in range(16):
        path = ens.trajectory(p)
        for k, i in enumerate(path.indices_at(obs)):
            assert list(ens.observed[p, k]) == list(path.states[i]), (p, k)


def test_tau_leaping_mean_with_many_paths(cuda):
    model = birth_death(20.0, 0.4)
    T = 3.0
    exact = 20.0 / 0.4 * (1.0 - math.exp(-0.4 * T))
    ens = simulate(model, [0], T, 100_000, seed=2, method="tau_leaping", leap=leap_options(epsilon=0.03))
    assert abs(ens.final_means()[0] - exact) < 0.3
    path = tau_leaping(model, [0], T, seed=2)
    assert path.times[-1] == pytest.approx(T)


def test_box_grows_until_no_path_leaves_it(cuda):
    ens = simulate(birth_death(100.0, 0.1), [0], 5.0, 1000, seed=9)
    assert ens.bounds[0] > 64 and np.all(ens.status == _lib.MK_OK)
    exact = 1000.0 * (1.0 - math.exp(-0.5))
    assert abs(ens.final_means()[0] - exact) < 5 * math.sqrt(exact / 1000)
    fixed = simulate(birth_death(100.0, 0.1), [0], 5.0, 64, seed=9, bounds=[100])
    assert np.all(fixed.status == _lib.MK_EOVERFLOW)
