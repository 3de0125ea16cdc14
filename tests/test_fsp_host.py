"""Non-GPU checks of the Krylov-FSP path: the golden fixtures the reference produced
(tests/golden/fsp_cases.npz) against closed-form answers, the propensity tabulation and box
indexing, and the C ABI's argument checks (which run before any device work)."""

import ctypes as C
import json
import math

import numpy as np
import pytest

import fsp_cases
from markovkit_b200 import _lib
from markovkit_b200.fsp import _Problem, box, krylov_fsp_options, tabulate
from markovkit_b200.inputs import fsp_batch_instances

GOLD = np.load(fsp_cases.__file__.replace("fsp_cases.py", "golden/fsp_cases.npz"))
META = json.loads(str(GOLD["meta"]))


def _dense(name: str, size: int) -> np.ndarray:
    p = np.zeros(size)
    p[GOLD[f"{name}/index"]] = GOLD[f"{name}/p"]
    return p


def test_fixture_pure_death_matches_closed_form():
    """tests/test_fsp.cpp:79-90: mean 5 e^-1 and extinction (1 - e^-1)^5, both within 1e-8."""
    p = _dense("pure_death_5", 6)
    assert META["pure_death_5"]["t"] == 1.0
    assert abs(np.dot(np.arange(6), p) - 5.0 * math.exp(-1.0)) < 1e-8
    assert abs(p[0] - (1.0 - math.exp(-1.0)) ** 5) < 1e-8


@pytest.mark.parametrize("k", [0, 1, 2])
def test_fixture_birth_death_is_poisson(k):
    """From the delta at 0 a birth-death law is Poisson with mean (b/d)(1 - e^{-d t})."""
    inst = fsp_batch_instances()[k]
    name = f"cfg_birth_death_{k}"
    n = inst["bounds"][0] + 1
    p = _dense(name, n)
    lam = inst["birth"] / inst["death"] * (1.0 - math.exp(-inst["death"] * inst["final_time"]))
    x = np.arange(n)
    pois = np.exp(x * math.log(lam) - lam - np.array([math.lgamma(v + 1.0) for v in x]))
    assert abs(p.sum() - 1.0) < 1e-12
    assert np.max(np.abs(p - pois)) < 1e-7


def test_fixture_metadata():
    assert META["zero_time"]["t"] == 0.0 and META["zero_time"]["support"] == 1
    assert META["no_reactions"]["support"] == 1
    assert META["birth_death_max_steps"]["t"] < 5.0  # stopped by max_steps
    for name, m in META.items():
        p = GOLD[f"{name}/p"]
        assert abs(p.sum() - 1.0) < 1e-12, name
        assert len(p) == m["support"]


def test_box_indexing_species_zero_most_significant():
    b = box([2, 3])
    st = b.states()
    assert st.shape == (12, 2)
    assert list(st[5]) == [1, 1]
    for i, x in enumerate(st):
        assert b.index(x) == i


def test_tabulate_vectorised_and_scalar_rates_agree():
    from markovkit_b200.fsp import reaction, reaction_network

    vec = reaction_network([reaction([1, -1], lambda x: 0.5 * x[:, 1] + x[:, 0])])
    scalar = reaction_network([reaction([1, -1], lambda x: 0.5 * x[1] + x[0])])
    ch1, r1 = tabulate(vec, box([3, 4]))
    ch2, r2 = tabulate(scalar, box([3, 4]))
    np.testing.assert_array_equal(ch1, ch2)
    np.testing.assert_array_equal(r1, r2)


def _create(problems):
    lib = _lib.load()
    arr = (_lib.FspProblem * len(problems))(*[p.c for p in problems])
    h = C.c_void_p()
    rc = lib.mk_fsp_batch_create(len(problems), arr, C.byref(h))
    return rc, lib.mk_last_error().decode()


def test_argument_errors_before_device_work():
    net, init, T, opt = fsp_cases.cases()["birth_death_two_layers"]
    bad = krylov_fsp_options(inside=opt.inside, krylov_dim=31)
    rc, msg = _create([_Problem(net, init, T, bad)])
    assert rc == _lib.MK_EINVAL and "krylov_dim" in msg
    rc, msg = _create([_Problem(net, [11], T, opt)])
    assert rc == _lib.MK_EINVAL and "initial" in msg
    rc, msg = _create([_Problem(net, init, -1.0, opt)])
    assert rc == _lib.MK_EINVAL and "final_time" in msg
    five = box([1, 1, 1, 1, 1])
    rc, msg = _create([_Problem(fsp_cases.reaction_network([]), [0] * 5, 1.0, krylov_fsp_options(inside=five))])
    assert rc == _lib.MK_EINVAL and "species" in msg
    with pytest.raises(ValueError):
        _Problem(net, init, T, krylov_fsp_options())  # no box region
    size = C.c_int64()
    assert _lib.load().mk_fsp_box_size(2, (C.c_int * 2)(40000, 40000), C.byref(size)) == _lib.MK_EOVERFLOW
    assert _lib.load().mk_fsp_box_size(2, (C.c_int * 2)(3, 4), C.byref(size)) == _lib.MK_OK
    assert size.value == 20


def test_regions_resolve_on_the_host():
    """box(bound) bounds every species once their count is known; the device FSP takes a box or
    everywhere() (None too) and refuses any other region before any device work."""
    from markovkit_b200.fsp import _first_box, _solve, box, everywhere

    assert box(7).resolved(3).bounds == [7, 7, 7]
    assert box([1, 2]).resolved(2).bounds == [1, 2]
    assert _first_box([0, 5]).bounds == [16, 21]
    net, init, T, opt = fsp_cases.cases()["birth_death_two_layers"]
    with pytest.raises(ValueError):
        _solve([(net, init, T, krylov_fsp_options(inside=lambda x: True))])
    assert isinstance(everywhere(), everywhere)
