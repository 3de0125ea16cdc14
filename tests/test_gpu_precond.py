"""The preconditioners beside the multigrid (num::jacobi_preconditioner, num::ilu0_preconditioner
and any host operator, examples/rdme_multigrid_benchmark.cpp:82-115) and generator::jumps(j)
(markovkit/generator.hpp:50-53), on a B200 through the C ABI.

- jumps(j): the reference's own jumps (tests/golden/jumps_golden.npz, make_jumps_golden.py)
  in the same order, targets exact, rates bitwise.
- ILU(0): the device factorisation and solves against the CPU restatement of oracle/ilu0.py
  (Saad Alg. 10.4) within 1e-12 relative (the device fuses each update into one fma).
- GMRES with each preconditioner converges to the multigrid-preconditioned solution (1e-8
  relative); a host operator computing the same d .* v as the Jacobi preconditioner takes the
  same iterations to the same bits.
"""

import json
from pathlib import Path

import numpy as np
import pytest

import markovkit_b200 as mk
from markovkit_b200 import _lib
from oracle.ilu0 import ilu0_factor, ilu0_solve

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "jumps_golden.npz"


def _model(spec):
    dim, cells = spec["dim"], spec["cells"]
    h = spec.get("h", 1.0 / cells)
    fam = spec["model"]
    if fam == "birth_death":
        birth, death = spec["birth"], spec["death"]
        diff = [spec["D"]]
        rx = [mk.local_reaction([1], lambda n, v: birth * v), mk.local_reaction([-1], lambda n, v: death * n[0])]
    elif fam == "annihilation":
        k = spec["k"]
        diff = [spec["D"], spec.get("D2", spec["D"])]
        rx = [mk.local_reaction([-1, -1], lambda n, v: k * n[0] * n[1] / v)]
    else:
        diff = [spec["D"]]
        rx = []
    dom = mk.voxel_domain(mk.grid([cells] * dim, [h] * dim), diff)
    model = mk.reaction_diffusion(dom, rx)
    caps = [int(c) for c in str(spec["cap"]).split(",")]
    box = mk.population_box(cells ** dim, caps)
    return dom, model, box


def test_jumps_match_reference(cuda):
    gold = np.load(GOLD)
    meta = json.loads(str(gold["meta"]))
    for name, m in meta.items():
        spec = m["spec"]
        dom, model, box = _model(spec)
        Q = mk.generator(box, model, spec.get("boundary", "absorbing"))
        first, to, rate = gold[f"{name}/first"].astype(np.int64), gold[f"{name}/to"], gold[f"{name}/rate"]
        assert Q.rows() == m["N"]
        total = 0
        for j in range(Q.rows()):
            js = Q.jumps(j)
            ref_to = to[first[j]:first[j + 1]].astype(np.int64)
            ref_rate = rate[first[j]:first[j + 1]]
            assert [e.to for e in js] == list(ref_to), (name, j)
            assert [e.rate for e in js] == list(ref_rate), (name, j)
            total += len(js)
        assert total == Q.n_jumps()


def test_jumps_block_tridiagonal_across_sectors(cuda):
    """tests/test_rdme.cpp:122-140: reactions change a total by at most one, and all three
    kinds of jump occur"""
    dom, model, box = _model(dict(dim=1, cells=2, h=1.0, cap="3", model="birth_death", birth=2.0, death=0.25, D=0.5))
    Q = mk.generator(box, model)
    assert Q.rows() == 10
    seen = set()
    for j in range(Q.rows()):
        for e in Q.jumps(j):
            change = box.sector_of(e.to) - box.sector_of(j)
            assert abs(change) <= 1
            seen.add(change)
    assert seen == {-1, 0, 1}
    # exit rate = in-space jumps + leak
    exits, leaks = Q.exit_rates().cpu().numpy(), Q.leak_rates().cpu().numpy()
    for j in range(Q.rows()):
        assert abs(sum(e.rate for e in Q.jumps(j)) + leaks[j] - exits[j]) <= 1e-14 * max(exits[j], 1.0)


def _system(spec, shift):
    dom, model, box = _model(spec)
    Q = mk.generator(box, model)
    return dom, box, Q, mk.shifted_generator(Q, shift)


CASES = {
    "birth_death_1d16_cap3": dict(dim=1, cells=16, cap="3", model="birth_death", birth=0.05, death=0.02, D=4.0),
    "annihilation_2d4": dict(dim=2, cells=4, cap="1,1", model="annihilation", k=10.0, D=1.0),
    "birth_death_3d2_cap2": dict(dim=3, cells=2, cap="2", model="birth_death", birth=0.05, death=0.02, D=4.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_ilu0_matches_oracle(cuda, name):
    import torch

    _, _, Q, A = _system(CASES[name], 0.5)
    Am = A.matrix()
    Am.sort_indices()
    M = mk.ilu0_preconditioner(Am)
    sched = M.schedule()
    assert sched["lower_levels"] >= 1 and sched["upper_levels"] >= 1 and sched["launches_per_apply"] >= 2
    lu, diag = ilu0_factor(Am.indptr, Am.indices, Am.data)
    rng = np.random.default_rng(7)
    for _ in range(2):
        v = rng.uniform(-1.0, 1.0, Q.rows())
        ref = ilu0_solve(Am.indptr, Am.indices, lu, diag, v)
        z = torch.zeros(Q.rows(), dtype=torch.float64, device=cuda)
        M.apply(torch.as_tensor(v, device=cuda), z)
        torch.cuda.synchronize()
        got = z.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)), name


@pytest.mark.parametrize("name", sorted(CASES))
def test_gmres_with_each_preconditioner(cuda, name):
    shift = 0.5
    dom, box, Q, A = _system(CASES[name], shift)
    n = Q.rows()
    b = 1.0 + 0.1 * np.cos(np.arange(n, dtype=np.float64))
    tol = 1e-10 * float(np.linalg.norm(b))
    opts = mk.gmres_options(tolerance=tol, max_iterations=2000, restart=50)

    def solve(M):
        x = np.zeros(n)
        r = mk.solver(A, M, opts).solve_host(b, x)
        assert r.converged, (name, r)
        return x, r

    x_mg, r_mg = solve(mk.sector_multigrid(dom, box, shift))
    d = 1.0 / (shift + Q.exit_rates().cpu().numpy())
    x_j, r_j = solve(mk.jacobi_preconditioner(d))
    x_ilu, r_ilu = solve(mk.ilu0_preconditioner(A.matrix()))
    scale = float(np.max(np.abs(x_mg)))
    for x in (x_j, x_ilu):
        assert np.max(np.abs(x - x_mg)) <= 1e-8 * scale, name
    # the same diagonal scaling as a host operator: same arithmetic, same iterates
    calls = []

    def host_apply(v):
        calls.append(1)
        return d * v

    x_h, r_h = solve(mk.host_preconditioner(n, host_apply))
    assert r_h.iterations == r_j.iterations and np.array_equal(x_h, x_j), name
    assert len(calls) >= r_h.iterations


def test_host_preconditioner_error_fails_the_solve(cuda):
    dom, box, Q, A = _system(CASES["birth_death_1d16_cap3"], 0.5)

    def broken(v):
        raise RuntimeError("no")

    s = mk.solver(A, mk.host_preconditioner(Q.rows(), broken), mk.gmres_options(tolerance=1e-10))
    with pytest.raises(_lib.MkError) as e:
        s.solve_host(np.ones(Q.rows()), np.zeros(Q.rows()))
    assert e.value.code == _lib.MK_EINVAL


def test_ilu0_zero_pivot_is_singular(cuda):
    import scipy.sparse as sp

    A = sp.csr_matrix((np.array([0.0, 1.0, 1.0, 0.0]), np.array([0, 1, 0, 1]), np.array([0, 2, 4])), shape=(2, 2))
    with pytest.raises(_lib.MkError) as e:
        mk.ilu0_preconditioner(A)
    assert e.value.code == _lib.MK_ESINGULAR
