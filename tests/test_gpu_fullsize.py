"""Resolvent solves at the benchmark's full sizes against the oracle, on a B200.

* The 2-D 32 x 32 two-particle annihilation box (1,050,625 states): the GPU solution of the
  seeded Dirichlet(1) right-hand side against the reference's own GMRES + sector_multigrid
  solution (tests/golden/full_annihilation_2d32.npz, made by make_full_golden.py).
* The 3-D 16^3 birth-death box of cap 2 (8,394,753 states): against the FP64 solution of the
  matrix-free CPU port of the reference's path (oracle/_ref/mf_port, run here on the host's
  cores; test_port_oracle.py checks it against the reference's own solutions first). The
  reference's containers need about 275 GB at this size.

Both precisions of the solver: FP64 GMRES(30) with the reference's FP64 multigrid, and FP64
flexible GMRES(30) with the FP32 multigrid of each smoother. Tolerances: 1e-10 relative true
residual, 1e-8 relative to the oracle's solution.
"""

import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import markovkit_b200 as mk
from markovkit_b200.inputs import dirichlet_rhs, uniform_rhs

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
PORT = ROOT / "oracle" / "_ref" / "mf_port"

PATHS = [("fp64", "jacobi", 4), ("fp32", "jacobi", 256), ("fp32", "gauss_seidel", 256), ("fp32", "ilu0", 256)]


def _problem(dim, cells, D, reactions, caps):
    dom = mk.voxel_domain(mk.grid([cells] * dim, [1.0 / cells] * dim), D)
    model = mk.reaction_diffusion(dom, reactions)
    box = mk.population_box(cells ** dim, caps)
    return dom, box, mk.generator(box, model, "absorbing")


def _solve(dev, dom, box, Q, shift, b, precision, smoother, coarsest):
    import torch

    A = mk.shifted_generator(Q, shift)
    M = mk.sector_multigrid(dom, box, shift, mk.multigrid_options(precision=precision, smoother=smoother,
                                                                  coarsest_size=coarsest))
    bt = torch.as_tensor(b, device=dev)
    bn = float(np.linalg.norm(b))
    s = mk.solver(A, M, mk.gmres_options(tolerance=1e-10 * bn, max_iterations=2000, restart=30,
                                         flexible=precision == "fp32"))
    x = torch.zeros_like(bt)
    res = s.solve(bt, x)
    y = torch.empty_like(x)
    A.apply(x, y)
    true_rel = float(torch.linalg.norm(bt - y)) / bn
    return x.cpu().numpy(), res, true_rel


@pytest.mark.parametrize("precision,smoother,coarsest", PATHS)
def test_annihilation_2d32_matches_reference(cuda, precision, smoother, coarsest):
    path = ROOT / "tests" / "golden" / "full_annihilation_2d32.npz"
    if not path.exists():
        pytest.skip("full_annihilation_2d32.npz not generated")
    ref = np.load(path)["x_mg"]
    dom, box, Q = _problem(2, 32, [1.0, 1.0], [mk.local_reaction([-1, -1], lambda n, v: 10.0 * n[0] * n[1] / v)],
                           [1, 1])
    assert box.size() == ref.size == 1050625
    b = dirichlet_rhs(1, box.size())
    x, res, true_rel = _solve(cuda, dom, box, Q, 1.0, b, precision, smoother, coarsest)
    assert res.converged and true_rel <= 1e-10
    assert float(np.linalg.norm(x - ref) / np.linalg.norm(ref)) <= 1e-8


@pytest.fixture(scope="module")
def birth_death_3d16_oracle():
    """the port's FP64 solution of the seeded uniform right-hand side (seed 2)"""
    if not PORT.exists():
        pytest.skip("oracle/_ref/mf_port is not built")
    with tempfile.TemporaryDirectory() as tmp:
        args = [str(PORT), "dim=3", "cells=16", "cap=2", "model=birth_death", "birth=0.05", "death=0.02", "D=1.0",
                "shift=0.5", "rhs=uniform", "seed=2", "tol=1e-10", "restart=30", f"threads={os.cpu_count() or 1}",
                "solves=1", f"out={tmp}"]
        proc = subprocess.run(args, capture_output=True, text=True, check=True, timeout=1800)
        meta = json.loads(proc.stdout.strip().splitlines()[-1])
        x = np.fromfile(Path(tmp) / "x_port.f64", dtype=np.float64)
    assert meta["converged"] and meta["true_rel_residual"] <= 1e-10
    return x


@pytest.mark.parametrize("precision,smoother,coarsest", PATHS)
def test_birth_death_3d16_matches_oracle(cuda, birth_death_3d16_oracle, precision, smoother, coarsest):
    ref = birth_death_3d16_oracle
    birth_death = [mk.local_reaction([1], lambda n, v: 0.05 * v), mk.local_reaction([-1], lambda n, v: 0.02 * n[0])]
    dom, box, Q = _problem(3, 16, [1.0], birth_death, [2])
    assert box.size() == ref.size == 8394753
    b = uniform_rhs(2, box.size())
    x, res, true_rel = _solve(cuda, dom, box, Q, 0.5, b, precision, smoother, coarsest)
    assert res.converged and true_rel <= 1e-10
    assert float(np.linalg.norm(x - ref) / np.linalg.norm(ref)) <= 1e-8
