"""The serving loop (mk_server_*) on a B200: results are the same alone and in the mix,
admission by HBM footprint evicts and waits as it should, and the FP32-multigrid served path
agrees with the all-FP64 path.

Tolerances: every solve reaches 1e-10 relative true residual (the north star's target); a
request's solution in the mix matches the same request served alone within 1e-8 relative
(both are 1e-10-residual solutions of one non-singular M-matrix system, and the multigrid
restriction sums with atomics, so they are not bitwise equal); the configuration-0 request
matches the reference's GMRES + sector_multigrid solution (tests/golden) within 1e-8 relative.
"""

import numpy as np
import pytest

import golden_cases as gc
import markovkit_b200 as mk
from markovkit_b200 import _lib
from markovkit_b200.inputs import dirichlet_rhs, uniform_rhs
from markovkit_b200.serve import server

pytestmark = pytest.mark.gpu


def _problem(dim, cells, caps, model, h=None):
    h = h if h is not None else 1.0 / cells
    D = [1.0] * len(caps)
    dom = mk.voxel_domain(mk.grid([cells] * dim, [h] * dim), D)
    if model == "annihilation":
        rx = [mk.local_reaction([-1, -1], lambda n, vol: 10.0 * n[0] * n[1] / vol)]
    else:
        rx = [mk.local_reaction([1], lambda n, vol: 0.05 * vol), mk.local_reaction([-1], lambda n, vol: 0.02 * n[0])]
    return mk.population_box(cells ** dim, caps), mk.reaction_diffusion(dom, rx)


PROBLEMS = {
    "cfg0": (1, 16, [3], "birth_death"),
    "ann2d8": (2, 8, [1, 1], "annihilation"),
    "bd3d4": (3, 4, [2], "birth_death"),
    "bd1d64": (1, 64, [2], "birth_death"),
}


def _requests():
    """(problem name, shift, seed, rhs kind) in submission order; shifts spread over [0.1, 10]"""
    reqs = [("cfg0", 0.5, 0, "uniform")]  # the configuration-0 request of the golden fixture
    rng = np.random.default_rng(4)
    names = list(PROBLEMS)
    for k in range(11):
        name = names[k % len(names)]
        shift = float(10 ** rng.uniform(-1, 1))
        reqs.append((name, shift, 100 + k, "dirichlet"))
    reqs.append(("bd3d4", reqs[3][1], 500, "dirichlet"))  # a second request on a resident key
    return reqs


def _rhs(kind, seed, n):
    return uniform_rhs(seed, n) if kind == "uniform" else dirichlet_rhs(seed, n)


def _serve(srv, reqs, spaces, at_once):
    pids = {name: srv.register(*spaces[name]) for name in PROBLEMS}
    out = []
    if at_once:
        tickets = [srv.submit(pids[n], s, _rhs(kind, seed, spaces[n][0].size())) for n, s, seed, kind in reqs]
        for t in tickets:
            out.append(srv.wait(t))
    else:
        for n, s, seed, kind in reqs:
            out.append(srv.wait(srv.submit(pids[n], s, _rhs(kind, seed, spaces[n][0].size()))))
    return out


@pytest.fixture(scope="module")
def spaces(cuda):
    return {name: _problem(*spec) for name, spec in PROBLEMS.items()}


@pytest.fixture(scope="module")
def alone(spaces):
    with server(slots=1, precision="fp32") as srv:
        return _serve(srv, _requests(), spaces, at_once=False)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_every_request_converges_alone(alone):
    for x, r in alone:
        assert r.status == _lib.MK_OK
        assert r.residual <= 1e-10


def test_same_alone_and_in_the_mix(spaces, alone):
    with server(slots=4, precision="fp32") as srv:
        mixed = _serve(srv, _requests(), spaces, at_once=True)
        st = srv.stats()
    assert st["completed"] == len(mixed)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (xa, ra), (xm, rm) in zip(alone, mixed):
        assert rm.status == _lib.MK_OK and rm.residual <= 1e-10
        assert _rel(xm, xa) <= 1e-8


def test_queued_requests_with_one_key_are_solved_together(spaces, alone):
    """One worker: while it solves a first request, four requests for one (problem, shift)
    queue up behind it and are then solved by one batched FGMRES; each matches its solve alone."""
    reqs = _requests()
    same = [r for r in reqs if r[0] == "cfg0"]  # cfg0 requests: (name, shift, seed, kind)
    key_shift = same[0][1]
    with server(slots=1, precision="fp32", batch=4) as srv:
        pids = {name: srv.register(*spaces[name]) for name in PROBLEMS}
        n = spaces["cfg0"][0].size()
        blocker = srv.submit(pids["bd1d64"], 1.0, dirichlet_rhs(77, spaces["bd1d64"][0].size()))
        tickets = [srv.submit(pids["cfg0"], key_shift, _rhs("dirichlet" if k else "uniform", 0 if k == 0 else 900 + k, n))
                   for k in range(4)]
        srv.wait(blocker)
        out = [srv.wait(t) for t in tickets]
    assert max(r.batched for _, r in out) >= 2
    # the first of them is the configuration-0 golden request: same solution as alone
    x0, r0 = out[0]
    assert r0.status == _lib.MK_OK and r0.residual <= 1e-10
    assert _rel(x0, alone[0][0]) <= 1e-8
    for x, r in out[1:]:
        assert r.status == _lib.MK_OK and r.residual <= 1e-10


def test_configuration_0_matches_the_reference(alone):
    c = gc.load("cfg0_birth_death_1d16")
    x, r = alone[0]
    assert _rel(x, c.data["x_mg"]) <= 1e-8


def test_fp64_path_agrees(spaces, alone):
    # the all-FP64 path, one request per solve (no batching), reference multigrid defaults
    with server(slots=2, precision="fp64", batch=1, coarsest_size=4) as srv:
        res = _serve(srv, _requests()[:5], spaces, at_once=True)
    for (x64, r64), (x32, r32) in zip(res, alone[:5]):
        assert r64.status == _lib.MK_OK and r64.residual <= 1e-10
        assert _rel(x64, x32) <= 1e-8


def test_admission_by_footprint(spaces, alone):
    reqs = _requests()
    with server(slots=3, precision="fp32") as probe:
        pids = {name: probe.register(*spaces[name]) for name in PROBLEMS}
        foot = {name: probe.footprint(pids[name]) for name in PROBLEMS}
    # room for the largest solver and a little more: new keys must evict or wait
    budget = max(foot.values()) + min(foot.values())
    with server(slots=3, precision="fp32", hbm_budget=budget) as srv:
        res = _serve(srv, reqs, spaces, at_once=True)
        st = srv.stats()
    assert st["resident_bytes"] <= budget
    assert st["evictions"] + st["memory_waits"] > 0
    for (xa, ra), (xm, rm) in zip(alone, res):
        assert rm.status == _lib.MK_OK
        assert _rel(xm, xa) <= 1e-8
    # a request larger than the whole budget is refused, not run (every footprint holds a fixed
    # 16 MiB besides the vectors, so 1 MiB is too small for any problem at any batch width)
    with server(slots=1, precision="fp32", hbm_budget=1 << 20) as small:
        pid = small.register(*spaces["bd1d64"])
        assert small.footprint(pid) > 1 << 20
        n = spaces["bd1d64"][0].size()
        t = small.submit(pid, 1.0, dirichlet_rhs(9, n))
        with pytest.raises(_lib.MkError):
            small.wait(t)
