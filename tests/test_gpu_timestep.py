"""Time stepping by repeated resolvents on a B200 (mk_solver_time_steps): backward Euler and
Crank-Nicolson with a Rannacher start, the paper driver's integrators
(rdme/cpp/rdme_full_multigrid.cpp:1173-1238), against direct sparse solves of the reference's
own assembled shift I - Q (tests/golden: Am) started from the same distribution.

Tolerances: every solve stops at 1e-10 relative residual, so after four steps the
distributions agree with the direct solves within 1e-8 relative (max norm); with a reflecting
boundary the total probability is conserved within 1e-9.
"""

import numpy as np
import pytest

import golden_cases as gc
import markovkit_b200 as mk

pytestmark = pytest.mark.gpu

CASES = ["cfg0_birth_death_1d16", "birth_death_2d4_reflecting", "annihilation_2d8"]
STEPS = 4


def _setup(c: gc.Case, precision: str):
    dom = mk.voxel_domain(mk.grid(c.dims, c.spacing), c.diffusivities)
    model = mk.reaction_diffusion(dom, [mk.local_reaction(ch, fn) for ch, fn in c.reactions])
    box = mk.population_box(int(np.prod(c.dims)), c.caps)
    Q = mk.generator(box, model, "absorbing" if c.absorbing else "reflecting")
    A = mk.shifted_generator(Q, c.shift)
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(precision=precision))
    opts = mk.gmres_options(max_iterations=2000, restart=30, flexible=precision == "fp32")
    return Q, mk.solver(A, M, opts)


def _direct_steps(c: gc.Case, p0: np.ndarray, integrator: str) -> np.ndarray:
    import scipy.sparse.linalg as spla

    A = c.csr("Am")
    lu = spla.splu(A.tocsc())
    s = c.shift
    p = p0.copy()
    solves = STEPS + (1 if integrator == "cn" else 0)
    for k in range(solves):
        rhs = 2.0 * s * p - A @ p if (integrator == "cn" and k >= 2) else s * p
        p = lu.solve(rhs)
    return p


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("integrator", ["be", "cn"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_time_steps_match_direct_solves(cuda, name, integrator, precision):
    import torch

    c = gc.load(name)
    _, sol = _setup(c, precision)
    p0 = c.data["b"] / np.sum(c.data["b"])
    p = torch.from_numpy(p0.copy()).to(cuda)
    res = sol.time_steps(p, STEPS, integrator, rel_tolerance=1e-10)
    assert len(res) == STEPS + (1 if integrator == "cn" else 0)
    assert all(r.converged for r in res)
    ref = _direct_steps(c, p0, integrator)
    got = p.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-8 * np.max(np.abs(ref))
    if not c.absorbing:
        assert abs(got.sum() - p0.sum()) <= 1e-9


def test_zero_steps_leave_p_unchanged(cuda):
    import torch

    c = gc.load("cfg0_birth_death_1d16")
    _, sol = _setup(c, "fp64")
    p0 = c.data["b"] / np.sum(c.data["b"])
    p = torch.from_numpy(p0.copy()).to(cuda)
    assert sol.time_steps(p, 0, "cn") == []
    np.testing.assert_array_equal(p.cpu().numpy(), p0)
