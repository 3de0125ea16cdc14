"""The assembled generator on a B200 (mk_generator_matrix, mk_generator_characteristic_matrix,
mk_generator_n_jumps; markovkit/generator.hpp:48, 84-107).

Against the reference: the CSR of Q.matrix() and of shifted_generator(Q, s).matrix() that
MarkovKit itself assembled for each golden fixture — identical row pointers and columns, values
within 1e-14 of their row's largest magnitude (entries are single rates or sums of a few,
in another order) — and n_jumps() equal to the reference's count.
At full size (the 2-D 32 x 32 annihilation box, 1,050,625 states): the assembled matrix
applied to a vector equals the matrix-free apply within 1e-13 relative (the reference checks
the same identity, tests/test_rdme.cpp:100-158), columns of Q sum to minus the leak rates,
and A = s I - Q entrywise.
"""

import numpy as np
import pytest

import golden_cases as gc
import markovkit_b200 as mk

pytestmark = pytest.mark.gpu
NAMES = gc.names()


def _setup(c: gc.Case):
    dom = mk.voxel_domain(mk.grid(c.dims, c.spacing), c.diffusivities)
    model = mk.reaction_diffusion(dom, [mk.local_reaction(ch, fn) for ch, fn in c.reactions])
    box = mk.population_box(int(np.prod(c.dims)), c.caps)
    return mk.generator(box, model, "absorbing" if c.absorbing else "reflecting")


def _same_csr(a, b, rtol):
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.indices, b.indices)
    scale = np.repeat(np.maximum.reduceat(np.abs(b.data), b.indptr[:-1]), np.diff(b.indptr))
    assert np.all(np.abs(a.data - b.data) <= rtol * scale)


@pytest.mark.parametrize("name", NAMES)
def test_matrix_equals_reference(cuda, name):
    c = gc.load(name)
    Q = _setup(c)
    Qm = Q.matrix()
    Am = mk.shifted_generator(Q, c.shift).matrix()
    assert Qm.has_sorted_indices and Am.has_sorted_indices
    _same_csr(Qm, c.csr("Qm"), 1e-14)
    _same_csr(Am, c.csr("Am"), 1e-14)
    assert Q.n_jumps() == int(c.ref["n_jumps"])


def test_device_arrays_match_host_copy(cuda):
    c = gc.load("annihilation_2d8")
    Q = _setup(c)
    m = Q.characteristic_matrix(c.shift, device=True)
    ptr, col, val = m.tensors()
    host = m.to_scipy()
    np.testing.assert_array_equal(ptr.cpu().numpy(), host.indptr)
    np.testing.assert_array_equal(col.cpu().numpy(), host.indices)
    np.testing.assert_array_equal(val.cpu().numpy(), host.data)
    assert m.size() == (c.n, host.nnz)


def test_full_size_properties(cuda):
    import scipy.sparse as sp
    import torch

    from markovkit_b200.inputs import uniform01

    dom = mk.voxel_domain(mk.grid([32, 32], [1 / 32, 1 / 32]), [1.0, 1.0])
    model = mk.reaction_diffusion(dom, [mk.local_reaction([-1, -1], lambda n, vol: 10.0 * n[0] * n[1] / vol)])
    box = mk.population_box(1024, [1, 1])
    Q = mk.generator(box, model, "absorbing")
    N = box.size()
    assert N == 1_050_625
    Qm = Q.matrix()
    x = uniform01(77, N)
    y = torch.empty(N, dtype=torch.float64, device=cuda)
    Q.apply(torch.from_numpy(x).to(cuda), y)
    ref = y.cpu().numpy()
    assert np.max(np.abs(Qm @ x - ref)) <= 1e-13 * np.max(np.abs(ref))
    # probability leaves Q's column j only through the leak: sum_i Q_ij = -leak_j
    _, leak = Q.exit_leak()
    colsum = np.asarray(Qm.sum(axis=0)).ravel()
    assert np.max(np.abs(colsum + leak.cpu().numpy())) <= 1e-12 * np.max(np.abs(Qm.diagonal()))
    s = 1.0
    Am = Q.characteristic_matrix(s)
    diff = (Am - (s * sp.identity(N, format="csr") - Qm)).tocsr()
    assert (abs(diff).max() if diff.nnz else 0.0) == 0.0
    # every row holds its diagonal, and no two jumps of this model join the same pair of states
    assert Q.n_jumps() == Qm.nnz - N
