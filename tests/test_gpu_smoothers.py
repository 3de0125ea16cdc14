"""The multigrid smoothers on a B200 against dense restatements.

The level operator A = shift I - Q_diffusion of configuration 0 (1-D, 16 voxels, box cap 3,
969 states) is assembled densely from the device's own matrix-free apply (one column per unit
vector); its checkerboard colouring (parity of sum over molecules of their voxel's
coordinate) is computed from the reference's enumeration of the states (tests/golden). Then:

  * the graph is bipartite in that colouring (no colour-0/colour-0 or colour-1/colour-1
    coupling), the property every colour-ordered smoother here relies on;
  * one red-black Gauss-Seidel pass pair equals the dense colour-ordered Gauss-Seidel sweep;
  * one ILU(0) sweep equals x + (L U)^-1 (b - A x) with the dense red-black ILU(0) factors,
    whose product agrees with A on A's sparsity pattern (the defining property of ILU(0)),
    all within 1e-12 relative;
  * multigrid-preconditioned GMRES with each smoother reaches 1e-10 relative true residual
    and the reference's solution within 1e-8 relative (tests/golden x_mg).
"""

import numpy as np
import pytest

import golden_cases as gc
import markovkit_b200 as mk

pytestmark = pytest.mark.gpu


def _case():
    c = gc.load("cfg0_birth_death_1d16")
    dom = mk.voxel_domain(mk.grid(c.dims, c.spacing), c.diffusivities)
    model = mk.reaction_diffusion(dom, [mk.local_reaction(ch, fn) for ch, fn in c.reactions])
    box = mk.population_box(int(np.prod(c.dims)), c.caps)
    return c, dom, model, box


def _dense_level(M, n, dev):
    import torch

    A = np.zeros((n, n))
    e = torch.zeros(n, dtype=torch.float64, device=dev)
    y = torch.empty_like(e)
    for j in range(n):
        e.zero_()
        e[j] = 1.0
        M.apply_system(0, e, y)
        A[:, j] = y.cpu().numpy()
    return A


def _colours(c):
    states = c.data["states"]  # n x V (one species), counts per voxel
    V = states.shape[1]
    parity = np.arange(V) % 2
    return (states @ parity) % 2


@pytest.fixture(scope="module")
def level(cuda):
    c, dom, model, box = _case()
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(smoother="ilu0"))
    n = box.size()
    A = _dense_level(M, n, cuda)
    return c, dom, box, A, _colours(c)


def test_level_operator_is_bipartite_in_the_state_colour(level):
    c, dom, box, A, col = level
    off = A - np.diag(np.diag(A))
    same = (col[:, None] == col[None, :])
    assert np.count_nonzero(off[same]) == 0
    assert np.count_nonzero(off) > 0


def _run_smoother(cuda, dom, box, shift, smoother, b, x):
    import torch

    M = mk.sector_multigrid(dom, box, shift, mk.multigrid_options(smoother=smoother))
    bt = torch.from_numpy(b).to(cuda)
    xt = torch.from_numpy(x.copy()).to(cuda)
    M.smooth(0, bt, xt)
    return xt.cpu().numpy()


def test_gauss_seidel_pass_pair_matches_dense(cuda, level):
    c, dom, box, A, col = level
    rng = np.random.default_rng(0)
    b, x = rng.random(A.shape[0]), rng.random(A.shape[0])
    got = _run_smoother(cuda, dom, box, c.shift, "gauss_seidel", b, x)
    ref = x.copy()
    d = np.diag(A)
    off = A - np.diag(d)
    for colour in (0, 1):
        idx = np.nonzero(col == colour)[0]
        ref[idx] = (b[idx] - off[idx] @ ref) / d[idx]
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_ilu0_sweep_matches_dense_factors(cuda, level):
    c, dom, box, A, col = level
    n = A.shape[0]
    R, B = np.nonzero(col == 0)[0], np.nonzero(col == 1)[0]
    d = np.diag(A)
    # red-black ILU(0): L = [I 0; A_BR D_R^-1 I], U = [D_R A_RB; 0 P_B]
    P = d[B] - np.einsum("ij,j,ji->i", A[np.ix_(B, R)], 1.0 / d[R], A[np.ix_(R, B)])
    L = np.eye(n)
    U = np.zeros((n, n))
    L[np.ix_(B, R)] = A[np.ix_(B, R)] / d[R][None, :]
    U[R, R] = d[R]
    U[np.ix_(R, B)] = A[np.ix_(R, B)]
    U[B, B] = P
    LU = L @ U
    pattern = A != 0
    assert np.max(np.abs((LU - A)[pattern])) <= 1e-12 * np.max(np.abs(A))
    rng = np.random.default_rng(1)
    b, x = rng.random(n), rng.random(n)
    ref = x + np.linalg.solve(LU, b - A @ x)
    got = _run_smoother(cuda, dom, box, c.shift, "ilu0", b, x)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("smoother", ["jacobi", "gauss_seidel", "ilu0"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_preconditioned_solve_matches_reference(cuda, smoother, precision):
    import torch

    c, dom, model, box = _case()
    Q = mk.generator(box, model, "absorbing")
    A = mk.shifted_generator(Q, c.shift)
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(smoother=smoother, precision=precision))
    b = torch.from_numpy(c.data["b"]).to(cuda)
    x = torch.zeros_like(b)
    bn = float(torch.linalg.norm(b))
    r = mk.gmres(A, M, b, x, mk.gmres_options(tolerance=1e-10 * bn, max_iterations=500, restart=30,
                                              flexible=precision == "fp32"))
    assert r.converged
    res = torch.empty_like(x)
    A.apply(x, res)
    assert float(torch.linalg.norm(b - res)) <= 1.0001e-10 * bn
    ref = c.data["x_mg"]
    assert np.linalg.norm(x.cpu().numpy() - ref) <= 1e-8 * np.linalg.norm(ref)
