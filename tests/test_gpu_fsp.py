"""GPU parity of batched Krylov FSP (the persistent kernel behind mk_fsp_batch_*) against the
reference's own solve_krylov_fsp (tests/golden/fsp_cases.npz, made by
tests/golden/make_fsp_golden.py), on a B200.

Both sides run the same algorithm on the same tabulated propensities; they differ in
summation order (block reductions against sequential sums, classical Gram-Schmidt with one
re-orthogonalisation against modified Gram-Schmidt, and the order of new states in the
support). Tolerances: final time within 1e-12 relative; each final probability within 1e-9
absolute of the reference's (the distributions carry the solver's 1e-8 tolerances, so a
rounding-level difference stays far below them); every state the reference keeps with
probability above 1e-9 is kept. Closed forms: the reference test's pure-death mean and
extinction probability within 1e-8 (tests/test_fsp.cpp:79-90), birth-death Poisson laws
within 1e-7.
"""

import dataclasses
import json
import math

import numpy as np
import pytest

import fsp_cases
from markovkit_b200 import _lib
from markovkit_b200.fsp import _Problem, fsp_batch, solve_krylov_fsp
from markovkit_b200.inputs import fsp_batch_instances

pytestmark = pytest.mark.gpu

GOLD = np.load(fsp_cases.__file__.replace("fsp_cases.py", "golden/fsp_cases.npz"))
META = json.loads(str(GOLD["meta"]))
P_TOL = 1e-9


def _ref_dense(name: str, size: int) -> np.ndarray:
    p = np.zeros(size)
    p[GOLD[f"{name}/index"]] = GOLD[f"{name}/p"]
    return p


@pytest.fixture(scope="module")
def golden_batch(cuda):
    cases = fsp_cases.cases()
    names = list(cases)
    b = fsp_batch([_Problem(*cases[n]) for n in names])
    b.run()
    out, res = b.results()
    return names, b, out, res


def _check_case(name, b, out, res, k):
    size = b.problems[k].region.size()
    got = out[b.offsets[k]: b.offsets[k] + size]
    ref = _ref_dense(name, size)
    t_ref = META[name]["t"]
    assert abs(res[k].time - t_ref) <= 1e-12 * max(1.0, abs(t_ref)), name
    assert np.max(np.abs(got - ref)) <= P_TOL, (name, float(np.max(np.abs(got - ref))))
    kept = ref > P_TOL
    assert np.all(got[kept] > 0.0), name
    return got


def test_golden_cases_in_one_batch(golden_batch):
    names, b, out, res = golden_batch
    for k, name in enumerate(names):
        _check_case(name, b, out, res, k)
        if name in ("birth_death_max_steps", "cfg_toggle_295_capped"):
            assert res[k].status == _lib.MK_ENOTCONV
        else:
            assert res[k].status == _lib.MK_OK, name


def test_reference_pure_death_through_the_single_call(cuda):
    """tests/test_fsp.cpp:79-90 through solve_krylov_fsp."""
    net, init, T, opt = fsp_cases.cases()["pure_death_5"]
    sol = solve_krylov_fsp(net, init, T, opt)
    assert sol.times[-1] == 1.0
    assert abs(sol.means()[-1, 0] - 5.0 * math.exp(-1.0)) < 1e-8
    last = sol.snapshots[-1].as_dict()
    assert abs(last[(0,)] - (1.0 - math.exp(-1.0)) ** 5) < 1e-8


@pytest.mark.parametrize("threads", [128, 256, 512])
def test_every_shape_gives_the_same_answer(golden_batch, threads):
    names, b, out, res = golden_batch
    for blocks in (1, 3, 0):
        b.set_shape(threads, blocks)
        b.run()
        out2, res2 = b.results()
        assert np.max(np.abs(out2 - out)) <= 1e-12
        for r1, r2 in zip(res, res2):
            assert r1.time == r2.time and r1.status == r2.status
    b.set_shape(512, 0)


def test_repeated_runs_are_bitwise_identical(golden_batch):
    names, b, out, res = golden_batch
    b.set_shape(512, 0)
    b.run()
    out2, _ = b.results()
    b.run()
    out3, _ = b.results()
    np.testing.assert_array_equal(out2, out3)


def test_autotune_keeps_results(golden_batch):
    names, b, out, res = golden_batch
    threads, blocks = b.autotune(sample=0)
    assert threads in (128, 256, 512) and blocks >= 1
    b.run()
    out2, _ = b.results()
    assert np.max(np.abs(out2 - out)) <= 1e-12


@pytest.fixture(scope="module")
def batch512(cuda):
    """all 512 instances of the batching workload in one launch, at most 2000 attempts each"""
    inst = fsp_batch_instances()
    probs = []
    for x in inst:
        o = fsp_cases.krylov_fsp_options(inside=fsp_cases.box(x["bounds"]), tolerance=x["tolerance"],
                                         max_steps=2000)
        probs.append(_Problem(fsp_cases.network_of(x), x["initial"], x["final_time"], o))
    b = fsp_batch(probs)
    b.run()
    out, res = b.results()
    return inst, b, out, res


def test_batching_workload_properties(batch512):
    """All 512 instances of the batching workload in one launch, with at most 2000 attempts
    each (toggles whose box cuts through a likely region need far more: their leak budget
    forces tiny steps, in the reference too). Every instance that finishes reaches t = 2 and
    every one keeps unit mass; birth-death laws are Poisson; the instances the reference ran
    agree with it."""
    inst, b, out, res = batch512
    finished = 0
    for k, x in enumerate(inst):
        assert res[k].status in (_lib.MK_OK, _lib.MK_ENOTCONV)
        if res[k].status == _lib.MK_OK:
            finished += 1
            assert abs(res[k].time - 2.0) < 1e-12
        else:
            assert x["family"] == "toggle" and res[k].attempts == 2000
        size = b.problems[k].region.size()
        p = out[b.offsets[k]: b.offsets[k] + size]
        assert abs(p.sum() - 1.0) < 1e-12
        if x["family"] == "birth_death":
            lam = x["birth"] / x["death"] * (1.0 - math.exp(-x["death"] * 2.0))
            n = np.arange(size)
            pois = np.exp(n * math.log(lam) - lam - np.array([math.lgamma(v + 1.0) for v in n]))
            assert np.max(np.abs(p - pois)) < 1e-7, k
    assert finished >= 470
    for k in (0, 1, 2, 256, 257, 258):
        fam = "birth_death" if k < 256 else "toggle"
        name = f"cfg_{fam}_{k}"
        size = b.problems[k].region.size()
        got = out[b.offsets[k]: b.offsets[k] + size]
        assert np.max(np.abs(got - _ref_dense(name, size))) <= P_TOL, name


BATCH_GOLD_PATH = fsp_cases.__file__.replace("fsp_cases.py", "golden/fsp_batch_golden.npz")


def test_batching_instances_match_reference(batch512):
    """33 instances of the 512-instance launch (the first 16 of each family and a toggle the
    reference itself stops at the attempt cap) against the reference's solve_krylov_fsp with the
    same cap (tests/golden/fsp_batch_golden.npz, made by make_fsp_batch_golden.py): final times
    within 1e-12, probabilities within 1e-9, for finished and capped instances alike."""
    import os

    if not os.path.exists(BATCH_GOLD_PATH):
        pytest.skip("fsp_batch_golden.npz not generated")
    gold = np.load(BATCH_GOLD_PATH)
    meta = json.loads(str(gold["meta"]))
    inst, b, out, res = batch512
    capped = 0
    for key, m in meta["instances"].items():
        k = int(key)
        size = b.problems[k].region.size()
        got = out[b.offsets[k]: b.offsets[k] + size]
        ref = np.zeros(size)
        ref[gold[f"{key}/index"]] = gold[f"{key}/p"]
        assert abs(res[k].time - m["t"]) <= 1e-12 * max(1.0, abs(m["t"])), k
        assert np.max(np.abs(got - ref)) <= P_TOL, (k, float(np.max(np.abs(got - ref))))
        if m["t"] < inst[k]["final_time"]:
            capped += 1
            assert res[k].status == _lib.MK_ENOTCONV and res[k].attempts == meta["max_steps"], k
        else:
            assert res[k].status == _lib.MK_OK, k
    assert len(meta["instances"]) >= 32 and capped >= 1


@pytest.mark.parametrize("name,big", [("birth_death_leaky_box", [400]), ("chain3", [40, 40, 40])])
def test_everywhere_matches_a_box_the_support_never_reaches(cuda, name, big):
    """everywhere() (the reference's default region): the device box grows on the species an
    expansion crossed until no expansion meets it; the support and probabilities then equal
    those of a box far beyond the support (which no expansion meets either)"""
    from markovkit_b200.fsp import box, everywhere

    net, init, T, opt = fsp_cases.cases()[name]
    grown = solve_krylov_fsp(net, init, T, dataclasses.replace(opt, inside=everywhere()))
    boxed = solve_krylov_fsp(net, init, T, dataclasses.replace(opt, inside=box(big)))
    a, b = grown.snapshots[-1], boxed.snapshots[-1]
    assert np.array_equal(a.states, b.states)
    assert np.max(np.abs(a.probabilities - b.probabilities)) <= 1e-14
    assert grown.times[-1] == boxed.times[-1] == T
    # the default (inside=None) is everywhere() too
    again = solve_krylov_fsp(net, init, T, dataclasses.replace(opt, inside=None))
    assert np.array_equal(again.snapshots[-1].probabilities, a.probabilities)


def test_clipped_reports_the_species_a_box_stopped(cuda):
    cases = fsp_cases.cases()
    names = ["birth_death_two_layers", "pure_death_5", "chain3"]
    b = fsp_batch([cases[n] for n in names])
    b.run()
    _, res = b.results(with_output=False)
    assert res[0].clipped == 1  # births out of box([10]): P(x > 10 at t = 0.5) > the tolerance
    assert res[1].clipped == 0  # deaths only
    assert res[2].clipped != 0 and res[2].clipped & ~0b111 == 0
