"""The full-operator multigrid (the paper driver's, rdme/cpp/rdme_full_multigrid.cpp:348-560,
819-850) on the GPU: every level is the whole box on a coarser grid, reactions included.

- One level is a dense solve of the whole box: one stationary cycle solves the system.
- As a solver of its own (V- and W-cycles, weighted Jacobi) and as a GMRES preconditioner, it
  reaches the solution of the sector-multigrid GMRES path (the system has one solution; both at
  1e-10 relative residual, so within 1e-6 relative: ||A^-1||_1 <= 1/s for s I - Q),
  on the paper's 1-D linear birth-death model (birth 2 vol, death n, D = 1, s = 0.5, cap 2) and on
  a 2-D two-species annihilation box.
- The K-cycle (two GCR steps per coarse visit, the paper driver's :851-878) reaches the same
  solution in no more cycles than the W-cycle.
- Gauss-Seidel runs over (sector colour class x checkerboard colour) passes: reactions couple
  states of one checkerboard colour, so the sectors they couple get different classes. It is
  deterministic and needs fewer cycles than Jacobi. ILU(0) smoothing and a K-cycle outside the
  full-operator FP64 hierarchy are refused."""

import numpy as np
import pytest

import markovkit_b200 as mk
from markovkit_b200 import _lib

pytestmark = pytest.mark.gpu


def _paper_model(cells, cap=2):
    dom = mk.voxel_domain(mk.grid([cells], [1.0 / cells]), [1.0])
    rx = [mk.local_reaction([1], lambda n, v: 2.0 * v), mk.local_reaction([-1], lambda n, v: 1.0 * n[0])]
    return dom, mk.reaction_diffusion(dom, rx), mk.population_box(cells, [cap])


def _annihilation(cells):
    dom = mk.voxel_domain(mk.grid([cells, cells], [1.0 / cells] * 2), [1.0, 1.0])
    rx = [mk.local_reaction([-1, -1], lambda n, v: 10.0 * n[0] * n[1] / v)]
    return dom, mk.reaction_diffusion(dom, rx), mk.population_box(cells * cells, [1, 1])


def _reference_solution(dom, model, box, shift, b):
    Q = mk.generator(box, model)
    A = mk.shifted_generator(Q, shift)
    x = np.zeros(box.size())
    tol = 1e-10 * float(np.linalg.norm(b))
    r = mk.solver(A, mk.sector_multigrid(dom, box, shift), mk.gmres_options(tolerance=tol, max_iterations=5000)).solve_host(b, x)
    assert r.converged
    return Q, A, x


def _rhs(n, seed=1):
    return np.random.default_rng(seed).uniform(0.0, 1.0, n)


def test_one_level_is_a_dense_solve(cuda):
    import torch

    dom, model, box = _paper_model(8)
    shift = 0.5
    M = mk.full_multigrid(model, box, shift, mk.multigrid_options(max_levels=1))
    assert M.max_levels() == 1
    Q = mk.generator(box, model)
    b = torch.as_tensor(_rhs(box.size()), device=cuda)
    x = torch.zeros_like(b)
    r = M.stationary(Q, b, x, tolerance=1e-12 * float(b.norm()), max_cycles=3)
    assert r.converged and r.iterations == 1


@pytest.mark.parametrize("cycles", [1, 2])
def test_stationary_iteration_reaches_the_solution(cuda, cycles):
    import torch

    dom, model, box = _paper_model(64)
    shift = 0.5
    b = _rhs(box.size(), 2)
    Q, A, x_ref = _reference_solution(dom, model, box, shift, b)
    M = mk.full_multigrid(model, box, shift, mk.multigrid_options(coarse_cycles=cycles))
    assert M.max_levels() == 7  # 64 -> 32 -> ... -> 1 voxel
    bt = torch.as_tensor(b, device=cuda)
    x = torch.zeros_like(bt)
    r = M.stationary(Q, bt, x, tolerance=1e-10 * float(np.linalg.norm(b)), max_cycles=500)
    assert r.converged, r
    got = x.cpu().numpy()
    assert np.max(np.abs(got - x_ref)) <= 1e-6 * np.max(np.abs(x_ref))


@pytest.mark.parametrize("case", ["paper_1d64", "annihilation_2d8"])
def test_preconditioner_reaches_the_solution(cuda, case):
    dom, model, box = _paper_model(64) if case == "paper_1d64" else _annihilation(8)
    shift = 0.5
    b = _rhs(box.size(), 3)
    Q, A, x_ref = _reference_solution(dom, model, box, shift, b)
    M = mk.full_multigrid(model, box, shift, mk.multigrid_options(coarse_cycles=2))
    x = np.zeros(box.size())
    r = mk.solver(A, M, mk.gmres_options(tolerance=1e-10 * float(np.linalg.norm(b)), max_iterations=500)).solve_host(b, x)
    assert r.converged
    assert np.max(np.abs(x - x_ref)) <= 1e-6 * np.max(np.abs(x_ref))


def test_ilu_smoother_is_refused(cuda):
    dom, model, box = _paper_model(8)
    with pytest.raises(_lib.MkError) as e:
        mk.full_multigrid(model, box, 0.5, mk.multigrid_options(smoother="ilu0"))
    assert e.value.code == _lib.MK_EINVAL


@pytest.mark.parametrize("case", ["paper_1d256", "annihilation_2d8"])
def test_multicolour_gauss_seidel(cuda, case):
    """Gauss-Seidel passes over (sector colour class x checkerboard colour): deterministic (two
    runs agree bit for bit), the same solution, and fewer W-cycles than weighted Jacobi"""
    import torch

    dom, model, box = _paper_model(256) if case == "paper_1d256" else _annihilation(8)
    shift = 0.5
    b = _rhs(box.size(), 5)
    Q, A, x_ref = _reference_solution(dom, model, box, shift, b)
    bt = torch.as_tensor(b, device=cuda)
    tol = 1e-10 * float(np.linalg.norm(b))
    its, xs = {}, []
    for sm in ("jacobi", "gauss_seidel", "gauss_seidel"):
        M = mk.full_multigrid(model, box, shift, mk.multigrid_options(coarse_cycles=2, smoother=sm))
        x = torch.zeros_like(bt)
        r = M.stationary(Q, bt, x, tolerance=tol, max_cycles=1000)
        assert r.converged, (sm, r)
        assert np.max(np.abs(x.cpu().numpy() - x_ref)) <= 1e-6 * np.max(np.abs(x_ref))
        its[sm] = r.iterations
        if sm == "gauss_seidel":
            xs.append(x.cpu().numpy())
    assert np.array_equal(xs[0], xs[1])
    assert its["gauss_seidel"] < its["jacobi"], its


@pytest.mark.parametrize("cells", [64, 256])
def test_k_cycle_reaches_the_solution(cuda, cells):
    import torch

    dom, model, box = _paper_model(cells)
    shift = 0.5
    b = _rhs(box.size(), 4)
    Q, A, x_ref = _reference_solution(dom, model, box, shift, b)
    bt = torch.as_tensor(b, device=cuda)
    tol = 1e-10 * float(np.linalg.norm(b))
    its = {}
    for kind, opts in (("w", dict(coarse_cycles=2)), ("k", dict(cycle_type="k"))):
        M = mk.full_multigrid(model, box, shift, mk.multigrid_options(**opts))
        x = torch.zeros_like(bt)
        r = M.stationary(Q, bt, x, tolerance=tol, max_cycles=1000)
        assert r.converged, (kind, r)
        assert np.max(np.abs(x.cpu().numpy() - x_ref)) <= 1e-6 * np.max(np.abs(x_ref))
        its[kind] = r.iterations
    assert its["k"] <= its["w"], its


def test_k_cycle_needs_the_full_fp64_hierarchy(cuda):
    dom, model, box = _paper_model(8)
    with pytest.raises(_lib.MkError):
        mk.full_multigrid(model, box, 0.5, mk.multigrid_options(cycle_type="k", precision="fp32"))
    with pytest.raises(_lib.MkError):
        mk.sector_multigrid(dom, box, 0.5, mk.multigrid_options(cycle_type="k"))

