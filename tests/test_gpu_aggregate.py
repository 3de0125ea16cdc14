"""The aggregate-block smoother (relaxation::aggregate_block, markovkit/rdme/multigrid.hpp:239-341)
against the reference's own sector_multigrid with that relaxation
(tests/golden/aggregate_golden.npz, made by make_aggregate_golden.py), on a B200.

Tolerances: one FP64 cycle within 1e-11 relative of the reference's (the blocks' residuals are
formed from rows instead of kept up to date by scatters, and dense inverses replace LU solves:
the same arithmetic in another order); FP32 cycles within 1e-5; GMRES(30) solutions with the
smoother at 1e-10 relative true residual within 1e-8 of the reference's. And the reference test's
claim (tests/test_rdme.cpp:214-217): a V-cycle with aggregate blocks reduces the residual more
than one with point Jacobi."""

import json
import math
from pathlib import Path

import numpy as np
import pytest

import markovkit_b200 as mk
from markovkit_b200.inputs import dirichlet_rhs, uniform_rhs

pytestmark = pytest.mark.gpu
GOLD_PATH = Path(__file__).resolve().parent / "golden" / "aggregate_golden.npz"


def _gold():
    if not GOLD_PATH.exists():
        pytest.skip("aggregate_golden.npz not generated")
    g = np.load(GOLD_PATH)
    return g, json.loads(str(g["meta"]))


def _problem(spec):
    dim, cells = int(spec["dim"]), int(spec["cells"])
    h = float(spec.get("h", 1.0 / cells))
    caps = [int(c) for c in str(spec["cap"]).split(",")]
    D = [float(spec["D"])] * len(caps)
    if spec["model"] == "birth_death":
        b, d = spec["birth"], spec["death"]
        rx = [mk.local_reaction([1], lambda n, v: b * v), mk.local_reaction([-1], lambda n, v: d * n[0])]
    elif spec["model"] == "annihilation":
        k = spec["k"]
        rx = [mk.local_reaction([-1, -1], lambda n, v: k * n[0] * n[1] / v)]
    else:
        rx = []
    dom = mk.voxel_domain(mk.grid([cells] * dim, [h] * dim), D)
    model = mk.reaction_diffusion(dom, rx)
    box = mk.population_box(cells ** dim, caps)
    rhs = dirichlet_rhs if spec["rhs"] == "dirichlet" else uniform_rhs
    return dom, model, box, float(spec["shift"]), rhs(int(spec["seed"]), box.size())


def _cases():
    if not GOLD_PATH.exists():
        return []
    return sorted(json.loads(str(np.load(GOLD_PATH)["meta"])))


@pytest.mark.parametrize("name", _cases())
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cycle_matches_reference(cuda, name, precision):
    import torch

    gold, meta = _gold()
    dom, _, box, shift, b = _problem(meta[name]["spec"])
    M = mk.sector_multigrid(dom, box, shift, mk.multigrid_options(smoother="aggregate_block", precision=precision))
    bt = torch.as_tensor(b, device=cuda)
    z = torch.empty_like(bt)
    M.apply(bt, z)
    ref = gold[f"{name}/Mb"]
    err = float(np.max(np.abs(z.cpu().numpy() - ref)) / np.max(np.abs(ref)))
    assert err <= (1e-11 if precision == "fp64" else 1e-5), err
    # the same cycle again: bitwise the same
    z2 = torch.empty_like(bt)
    M.apply(bt, z2)
    assert torch.equal(z, z2)


@pytest.mark.parametrize("name", _cases())
def test_solution_matches_reference(cuda, name):
    import torch

    gold, meta = _gold()
    dom, model, box, shift, b = _problem(meta[name]["spec"])
    Q = mk.generator(box, model, "absorbing")
    A = mk.shifted_generator(Q, shift)
    M = mk.sector_multigrid(dom, box, shift, mk.multigrid_options(smoother="aggregate_block"))
    bn = float(np.linalg.norm(b))
    s = mk.solver(A, M, mk.gmres_options(tolerance=1e-10 * bn, max_iterations=1000, restart=30))
    bt = torch.as_tensor(b, device=cuda)
    x = torch.zeros_like(bt)
    r = s.solve(bt, x)
    y = torch.empty_like(x)
    A.apply(x, y)
    assert r.converged and float(torch.linalg.norm(bt - y)) / bn <= 1e-10
    ref = gold[f"{name}/x_mg"]
    assert float(np.linalg.norm(x.cpu().numpy() - ref) / np.linalg.norm(ref)) <= 1e-8


def test_aggregate_blocks_beat_point_jacobi(cuda):
    """population_multigrid(domain 1-D 8 voxels h = 1, D = 1, totals {2}, shift 1): one cycle
    from b_i = 0.25 + sin(i) leaves a smaller residual with aggregate blocks than with Jacobi,
    and Jacobi's is below the initial one (tests/test_rdme.cpp:197-217)"""
    import torch

    dom = mk.voxel_domain(mk.grid([8], [1.0]), [1.0])
    sector = mk.population_sector(8, [2])
    Q = mk.generator(sector, mk.reaction_diffusion(dom, []), "absorbing")
    A = mk.shifted_generator(Q, 1.0)
    assert sector.size() == 36
    b = torch.tensor([0.25 + math.sin(i) for i in range(36)], dtype=torch.float64, device=cuda)

    def residual(smoother):
        M = mk.sector_multigrid(dom, sector, 1.0, mk.multigrid_options(smoother=smoother))
        x = torch.empty_like(b)
        M.apply(b, x)
        y = torch.empty_like(b)
        A.apply(x, y)
        return float(torch.sum((b - y) ** 2))

    initial = float(torch.sum(b * b))
    jacobi = residual("jacobi")
    block = residual("aggregate_block")
    assert jacobi < initial and block < jacobi
