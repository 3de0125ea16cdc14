"""solve_adaptive_fsp (markovkit/fsp.hpp:123-188) on the GPU against the reference's own runs
(tests/golden/fsp_adaptive_golden.npz, made by make_fsp_adaptive_golden.py), in one batched
launch beside Krylov-FSP instances.

Both sides expand, propagate with expv on the reflecting generator of the support, prune with
the same selection (the least likely states, ties by support order) and renormalise; they sum
in another order. Tolerances: final time within 1e-12 relative, each final probability within
1e-9 absolute. And the reference test's check (tests/test_fsp.cpp:68-77): the birth-death mean
within 0.1 of (lambda / mu)(1 - e^{-mu t})."""

import json
import math
from pathlib import Path

import numpy as np
import pytest

from markovkit_b200 import _lib
from markovkit_b200.fsp import _Problem, adaptive_fsp_options, box, fsp_batch, krylov_fsp_options, solve_adaptive_fsp
from markovkit_b200.fsp_models import birth_death, toggle

pytestmark = pytest.mark.gpu
GOLD_PATH = Path(__file__).resolve().parent / "golden" / "fsp_adaptive_golden.npz"
P_TOL = 1e-9


def _network(c):
    if c["family"] == "birth_death":
        return birth_death(c["birth"], c["death"])
    return toggle(c["a1"], c["a2"], c["n1"], c["n2"])


@pytest.fixture(scope="module")
def adaptive_batch(cuda):
    if not GOLD_PATH.exists():
        pytest.skip("fsp_adaptive_golden.npz not generated")
    gold = np.load(GOLD_PATH)
    meta = json.loads(str(gold["meta"]))
    names = sorted(meta)
    probs = []
    for n in names:
        c = meta[n]["case"]
        probs.append(_Problem(_network(c), c["initial"], c["T"],
                              adaptive_fsp_options(inside=box(c["bounds"]), **c["options"])))
    # a Krylov-FSP instance in the same launch: the two methods share the kernel
    probs.append(_Problem(birth_death(5.0, 0.2), [0], 1.0, krylov_fsp_options(inside=box([80]), tolerance=1e-8)))
    b = fsp_batch(probs)
    b.run()
    out, res = b.results()
    return gold, meta, names, b, out, res


def test_adaptive_matches_reference(adaptive_batch):
    gold, meta, names, b, out, res = adaptive_batch
    for k, name in enumerate(names):
        m = meta[name]
        size = b.problems[k].region.size()
        got = out[b.offsets[k]: b.offsets[k] + size]
        ref = np.zeros(size)
        ref[gold[f"{name}/index"]] = gold[f"{name}/p"]
        assert abs(res[k].time - m["t"]) <= 1e-12 * max(1.0, abs(m["t"])), name
        assert np.max(np.abs(got - ref)) <= P_TOL, (name, float(np.max(np.abs(got - ref))))
        assert abs(got.sum() - 1.0) < 1e-12, name
        finished = m["t"] >= m["case"]["T"]
        assert res[k].status == (_lib.MK_OK if finished else _lib.MK_ENOTCONV), name
    # the Krylov-FSP instance of the same launch: a Poisson law with mean (b / d)(1 - e^{-d t})
    k = len(names)
    lam = 5.0 / 0.2 * (1.0 - math.exp(-0.2))
    n = np.arange(81)
    pois = np.exp(n * math.log(lam) - lam - np.array([math.lgamma(v + 1.0) for v in n]))
    assert np.max(np.abs(out[b.offsets[k]: b.offsets[k] + 81] - pois)) < 1e-6


def test_reference_adaptive_birth_death_mean(cuda):
    sol = solve_adaptive_fsp(birth_death(5.0, 0.1), [0], 2.0, adaptive_fsp_options(inside=box([100]), step_scale=0.1))
    mean = float(sol.means()[-1][0])
    exact = (5.0 / 0.1) * (1.0 - math.exp(-0.1 * 2.0))
    assert abs(mean - exact) < 0.1
    assert len(sol.times) > 1 and sol.times[-1] == 2.0


def test_sampled_expansion_is_refused():
    with pytest.raises(ValueError):
        adaptive_fsp_options(inside=box([10]), sampled_expansion=True)._c()
