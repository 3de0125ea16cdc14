"""Failure handling of the resolvent path on a B200, made on the host (no GPU fault is
provoked): a non-finite right-hand side ends GMRES with MK_ENAN; a zero right-hand side
converges at iteration 0; a queued server request can be cancelled (MK_ECANCELED) and a bounded
wait on an unfinished request gives up with MK_ETIMEOUT while the request completes later."""

import numpy as np
import pytest

import markovkit_b200 as mk
from markovkit_b200 import _lib
from markovkit_b200.serve import server

pytestmark = pytest.mark.gpu


def _system(shift=0.5):
    dom = mk.voxel_domain(mk.grid([16], [1.0 / 16]), [4.0])
    rx = [mk.local_reaction([1], lambda n, v: 0.05 * v), mk.local_reaction([-1], lambda n, v: 0.02 * n[0])]
    model = mk.reaction_diffusion(dom, rx)
    box = mk.population_box(16, [3])
    Q = mk.generator(box, model)
    return dom, model, box, Q, mk.shifted_generator(Q, shift)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_rhs_is_enan(cuda, bad):
    dom, model, box, Q, A = _system()
    M = mk.sector_multigrid(dom, box, 0.5)
    b = np.ones(Q.rows())
    b[17] = bad
    for pre in (M, None):
        s = mk.solver(A, pre, mk.gmres_options(tolerance=1e-10))
        with pytest.raises(_lib.MkError) as e:
            s.solve_host(b, np.zeros(Q.rows()))
        assert e.value.code == _lib.MK_ENAN


def test_zero_rhs_converges_at_iteration_zero(cuda):
    dom, model, box, Q, A = _system()
    M = mk.sector_multigrid(dom, box, 0.5)
    x = np.zeros(Q.rows())
    r = mk.solver(A, M, mk.gmres_options(tolerance=0.0)).solve_host(np.zeros(Q.rows()), x)
    assert r.converged and r.iterations == 0 and r.residual == 0.0
    assert not np.any(x)


def test_server_nonfinite_rhs_is_enan(cuda):
    dom, model, box, Q, A = _system()
    with server(slots=1, batch=1) as srv:
        p = srv.register(box, model)
        b = np.ones(Q.rows())
        b[3] = np.nan
        t = srv.submit(p, 0.5, b)
        with pytest.raises(_lib.MkError) as e:
            srv.wait(t)
        assert e.value.code == _lib.MK_ENAN
        # the server goes on serving
        x, r = srv.wait(srv.submit(p, 0.5, np.ones(Q.rows())))
        assert r.status == _lib.MK_OK


def _slow_problem():
    """a box large enough that building its resident solver and solving keeps the only slot
    busy for a while (3D 16^3 voxels, birth-death, cap 2: 8.4M states)"""
    dom = mk.voxel_domain(mk.grid([16, 16, 16], [1.0 / 16] * 3), [1.0])
    rx = [mk.local_reaction([1], lambda n, v: 0.05 * v), mk.local_reaction([-1], lambda n, v: 0.02 * n[0])]
    return mk.reaction_diffusion(dom, rx), mk.population_box(16 ** 3, [2])


def test_server_cancel_and_timeout(cuda):
    model, box = _slow_problem()
    n = box.size()
    with server(slots=1, batch=1, precision="fp32", smoother="gauss_seidel") as srv:
        p = srv.register(box, model)
        b = np.ones(n)
        first = srv.submit(p, 0.5, b)
        queued = srv.submit(p, 0.7, b)
        to_cancel = srv.submit(p, 0.9, b)
        srv.cancel(to_cancel)
        with pytest.raises(_lib.MkError) as e:
            srv.cancel(to_cancel)  # no longer queued
        assert e.value.code == _lib.MK_EINVAL
        _, r = srv.wait(to_cancel, allow=(_lib.MK_ECANCELED,))
        assert r.status == _lib.MK_ECANCELED
        # the second request waits behind the first: a zero-length wait gives up
        with pytest.raises(_lib.MkError) as e:
            srv.wait(queued, timeout_ms=0.0)
        assert e.value.code == _lib.MK_ETIMEOUT
        x1, r1 = srv.wait(first)
        x2, r2 = srv.wait(queued, timeout_ms=600_000.0)
        assert r1.status == _lib.MK_OK and r2.status == _lib.MK_OK
        assert np.all(np.isfinite(x1)) and np.all(np.isfinite(x2))
        assert srv.stats()["completed"] == 2
