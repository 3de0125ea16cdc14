"""Batched resolvent solves on a B200: up to four right-hand sides of one system advanced in
lockstep by flexible GMRES, with one batched generator apply and one batched multigrid cycle
per step for all of them.

Checks: a batched multigrid cycle equals the single-column cycle column by column (FP64
hierarchies: within 1e-12 relative, the restriction sums with atomics); a batched operator
apply equals the single one bit for bit; every column of a batched solve reaches its 1e-10
relative true residual and matches the same right-hand side solved alone within 1e-8 relative,
and the configuration-0 column matches the reference's solution (tests/golden) within 1e-8.
"""

import numpy as np
import pytest

import golden_cases as gc
import markovkit_b200 as mk
from markovkit_b200.inputs import dirichlet_rhs

pytestmark = pytest.mark.gpu


def _problem(name):
    c = gc.load(name)
    dom = mk.voxel_domain(mk.grid(c.dims, c.spacing), c.diffusivities)
    model = mk.reaction_diffusion(dom, [mk.local_reaction(ch, fn) for ch, fn in c.reactions])
    box = mk.population_box(int(np.prod(c.dims)), c.caps)
    Q = mk.generator(box, model, "absorbing" if c.absorbing else "reflecting")
    return c, dom, box, Q


def _rhs(c, n, k):
    return c.data["b"] if k == 0 else dirichlet_rhs(300 + k, n)


@pytest.mark.parametrize("name", ["cfg0_birth_death_1d16", "annihilation_2d8", "birth_death_3d4_cap2"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batched_cycle_equals_single_cycles(cuda, name, precision):
    import torch

    c, dom, box, Q = _problem(name)
    n = box.size()
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(precision=precision, batch=4))
    nb = 3
    ld = n + 5  # columns need not be packed
    B = torch.zeros(nb, ld, dtype=torch.float64, device=cuda)
    for k in range(nb):
        B[k, :n] = torch.from_numpy(_rhs(c, n, k))
    X = torch.zeros_like(B)
    lib = mk.api.load()
    mk.api.check(lib.mk_multigrid_apply_batch(M._h, mk.api._ptr(B), ld, mk.api._ptr(X), ld, nb,
                                              mk.api._stream(None)))
    # FP64: only the order of the restriction's atomic sums differs; FP32: float rounding
    tol = 1e-12 if precision == "fp64" else 1e-5
    for k in range(nb):
        x = torch.zeros(n, dtype=torch.float64, device=cuda)
        M.apply(B[k, :n].contiguous(), x)
        ref = x.cpu().numpy()
        assert np.max(np.abs(X[k, :n].cpu().numpy() - ref)) <= tol * np.max(np.abs(ref))
    # the batched generator apply is the single apply, column by column, bit for bit
    Y = torch.zeros_like(B)
    mk.api.check(lib.mk_generator_apply_shifted_batch(Q._h, c.shift, mk.api._ptr(B), mk.api._ptr(Y), ld, nb,
                                                      mk.api._stream(None)))
    for k in range(nb):
        y = torch.empty(n, dtype=torch.float64, device=cuda)
        Q.apply_shifted(c.shift, B[k, :n].contiguous(), y)
        assert torch.equal(Y[k, :n], y)


@pytest.mark.parametrize("name", ["cfg0_birth_death_1d16", "annihilation_2d8", "birth_death_3d4_cap2", "annihilation_1d6_cap2"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batched_solve_matches_single_solves(cuda, name, precision):
    import torch

    c, dom, box, Q = _problem(name)
    n = box.size()
    A = mk.shifted_generator(Q, c.shift)
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(precision=precision, batch=4))
    nb = 4
    B = torch.stack([torch.from_numpy(_rhs(c, n, k)) for k in range(nb)]).to(cuda).contiguous()
    X = torch.zeros_like(B)
    tols = [1e-10 * float(torch.linalg.norm(B[k])) for k in range(nb)]
    bs = mk.batch_solver(A, M, mk.gmres_options(max_iterations=2000, restart=30), width=4)
    res = bs.solve(B, X, tols)
    Msingle = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(precision=precision))
    for k in range(nb):
        assert res[k].converged, (k, res[k])
        r = torch.empty(n, dtype=torch.float64, device=cuda)
        A.apply(X[k].contiguous(), r)
        assert float(torch.linalg.norm(B[k] - r)) <= 1.0001 * tols[k]
        x1 = torch.zeros(n, dtype=torch.float64, device=cuda)
        r1 = mk.gmres(A, Msingle, B[k].contiguous(), x1,
                      mk.gmres_options(tolerance=tols[k], max_iterations=2000, restart=30, flexible=True))
        assert r1.converged
        assert float(torch.linalg.norm(X[k] - x1) / torch.linalg.norm(x1)) <= 1e-8
    if name.startswith("cfg0"):
        ref = c.data["x_mg"]
        assert np.linalg.norm(X[0].cpu().numpy() - ref) <= 1e-8 * np.linalg.norm(ref)


def test_partial_batch_and_uneven_convergence(cuda):
    """Fewer columns than the width, and columns that converge at different steps (one
    right-hand side is already solved by its initial guess)."""
    import torch

    c, dom, box, Q = _problem("annihilation_2d8")
    n = box.size()
    A = mk.shifted_generator(Q, c.shift)
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(precision="fp32", batch=4))
    B = torch.stack([torch.from_numpy(_rhs(c, n, k)) for k in range(3)]).to(cuda).contiguous()
    X = torch.zeros_like(B)
    # column 2 starts from a converged solution
    x2 = torch.zeros(n, dtype=torch.float64, device=cuda)
    tol2 = 1e-10 * float(torch.linalg.norm(B[2]))
    mk.gmres(A, M, B[2].contiguous(), x2, mk.gmres_options(tolerance=tol2 * 0.5, max_iterations=2000, flexible=True))
    X[2] = x2
    tols = [1e-10 * float(torch.linalg.norm(B[k])) for k in range(3)]
    bs = mk.batch_solver(A, M, mk.gmres_options(max_iterations=2000, restart=30), width=4)
    res = bs.solve(B, X, tols)
    assert all(r.converged for r in res)
    assert res[2].iterations == 0
    assert res[0].iterations > 0 and res[1].iterations > 0
