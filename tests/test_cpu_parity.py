"""Non-GPU parity: the product's shared host/device row logic (state indexing, generator
gather, multigrid transfer), run on the CPU through tests/cpu/emulate.cpp, against the
golden vectors the reference produced (tests/golden/)."""

import numpy as np
import pytest

import cpu_emulator as emu
import golden_cases as gc

NAMES = gc.names()


@pytest.mark.parametrize("name", [n for n in NAMES if "states" in gc.load(n).data])
def test_state_indexing_bit_exact(name):
    c = gc.load(name)
    S = len(c.caps)
    states, ranks = emu.states(int(np.prod(c.dims)), c.caps, is_box=True)
    ref_states = c.data["states"]
    assert states.shape == ref_states.shape
    np.testing.assert_array_equal(states, ref_states)  # unrank == enumeration order
    np.testing.assert_array_equal(ranks, np.arange(len(ranks)))  # rank(state[i]) == i
    np.testing.assert_array_equal(c.data["find"].astype(np.int64), np.arange(len(ranks)))
    assert S >= 1


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("csr", [False, True], ids=["grid", "csr"])
def test_generator_rows_match_reference(name, csr):
    c = gc.load(name)
    out = emu.generator(c.dim, c.dims, c.spacing, c.diffusivities, c.reactions, c.caps, True, c.absorbing, c.shift, c.data["x"], csr=csr)
    # exit and leak rates: sums of the same positive terms, in another order
    np.testing.assert_allclose(out["exit"], c.data["exit"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(out["leak"], c.data["leak"], rtol=1e-14, atol=0)
    # a single FP64 generator apply within 1e-13 relative (max-norm)
    for key in ("Qx", "Ax"):
        ref = c.data[key]
        err = np.max(np.abs(out[key] - ref)) / np.max(np.abs(ref))
        assert err < 1e-13, (key, err)


@pytest.mark.parametrize("name", [n for n in NAMES if any(k.endswith("_Pc") for k in gc.load(n).data)])
def test_transfer_matches_reference(name):
    c = gc.load(name)
    for key in sorted(k for k in c.data if k.endswith("_Pc")):
        k = int(key[len("sector"):-3])
        totals_list = None
        # the box's sector k: recover its totals from the mixed-radix order
        caps = c.caps
        rem, totals_list = k, []
        for cap in reversed(caps):
            totals_list.append(rem % (cap + 1))
            rem //= cap + 1
        totals = list(reversed(totals_list))
        Pc, Rg = emu.transfer(c.dim, c.dims, c.spacing, totals, c.data[f"sector{k}_c"], c.data[f"sector{k}_g"])
        np.testing.assert_allclose(Pc, c.data[f"sector{k}_Pc"], rtol=1e-13, atol=1e-16)
        np.testing.assert_allclose(Rg, c.data[f"sector{k}_Rg"], rtol=1e-13, atol=1e-15)


def _same_csr(a, b, rtol):
    """identical sparsity (row pointers and sorted columns), values within rtol of the largest
    magnitude of their row"""
    a = a.tocsr()
    b = b.tocsr()
    a.sort_indices()
    b.sort_indices()
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.indices, b.indices)
    scale = np.repeat(np.maximum.reduceat(np.abs(b.data), b.indptr[:-1]) if b.nnz else np.zeros(0),
                      np.diff(b.indptr))
    assert np.all(np.abs(a.data - b.data) <= rtol * scale), np.max(np.abs(a.data - b.data) / scale)


@pytest.mark.parametrize("name", NAMES)
def test_reference_matrix_is_its_apply(name):
    """the oracle's own pin: the reference's assembled Q and shift I - Q reproduce its matrix-free
    apply (tests/test_rdme.cpp:100-158 checks the same), and A = shift I - Q entrywise"""
    c = gc.load(name)
    Qm, Am = c.csr("Qm"), c.csr("Am")
    x = c.data["x"]
    for m, key in ((Qm, "Qx"), (Am, "Ax")):
        ref = c.data[key]
        assert np.max(np.abs(m @ x - ref)) <= 1e-14 * np.max(np.abs(ref))
    diff = (Am - (c.shift * _eye(c.n) - Qm)).tocsr()
    assert (abs(diff).max() if diff.nnz else 0.0) <= 1e-15 * abs(Am).max()
    # one entry per jump before equal positions merge: nnz <= N + n_jumps
    assert Qm.nnz <= c.n + int(c.ref["n_jumps"])


def _eye(n):
    import scipy.sparse as sp

    return sp.identity(n, format="csr")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("csr", [False, True], ids=["grid", "csr"])
def test_assembled_rows_match_reference_matrix(name, csr):
    """the rows the device assembly writes (diagonal, then one entry per in-jump), merged like
    num::spmat::from_triplets, equal the reference's matrix() and characteristic_matrix()"""
    c = gc.load(name)
    args = (c.dim, c.dims, c.spacing, c.diffusivities, c.reactions, c.caps, True, c.absorbing)
    Q = emu.matrix(*args, shift=0.0, sign=1.0, csr=csr)
    A = emu.matrix(*args, shift=c.shift, sign=-1.0, csr=csr)
    _same_csr(Q, c.csr("Qm"), 1e-14)
    _same_csr(A, c.csr("Am"), 1e-14)


@pytest.mark.parametrize("dim,cells", [(1, 7), (2, 6), (3, 3)])
def test_stencil_rows_bit_identical(dim, cells):
    """diffusion-only rows of one molecule per species (the multigrid level operators of
    two-species boxes of cap 1) take visit_row's stencil path on grids; it must give exactly
    the general visit's exit rates and applies, and agree with the neighbour-list path"""
    dims, h = [cells] * dim, [1.0 / cells] * dim
    D, caps, x = [0.7, 1.9], [1, 1], None
    outs = {}
    for mode in (0, 2, 1):  # stencil, general grid visit, neighbour lists
        n = len(emu.generator(dim, dims, h, D, [], caps, True, True, 0.5, None, csr=mode)["exit"])
        if x is None:
            x = np.sin(0.37 * np.arange(n)) + 1.5
        outs[mode] = emu.generator(dim, dims, h, D, [], caps, True, True, 0.5, x, csr=mode)
    for key in ("exit", "leak", "Qx", "Ax"):
        np.testing.assert_array_equal(outs[0][key], outs[2][key])
        np.testing.assert_allclose(outs[0][key], outs[1][key], rtol=1e-14, atol=1e-12)


def _birth_death(b=0.05, d=0.02):
    return [([1], lambda n, v: b * v), ([-1], lambda n, v: d * n[0])]


@pytest.mark.parametrize(
    "dim,cells,D,reactions,caps,absorbing",
    [
        (1, 16, [1.0], _birth_death(), [3], True),          # the 16-voxel birth-death box of cap 3
        (1, 9, [0.8], _birth_death(2.0, 1.0), [4], False),  # cap 4, reflecting, odd grid
        (2, 5, [1.3], _birth_death(), [2], True),
        (3, 4, [1.0], _birth_death(), [2], True),           # a small copy of the 16^3 box of cap 2
        (3, 3, [0.5], [], [2], True),                        # a multigrid level operator
        (2, 6, [1.0, 1.0], [([-1, -1], lambda n, v: 10.0 * n[0] * n[1] / v)], [1, 1], True),
        (3, 3, [0.7, 1.9], [], [1, 1], True),
        (1, 12, [1.0], [], [4], True),
    ],
)
def test_stencil_forms_equal_general_visit(dim, cells, D, reactions, caps, absorbing):
    """The stencil row kernel's forms (closed-form unranking, voxel masks, closed-form source
    ranks) give every light row the same in-jumps, rates, exit and leak bits and colour as the
    general row visit, in the same order, so the two kernels agree bit for bit."""
    dims, h = [cells] * dim, [1.0 / cells] * dim
    rows = emu.stencil_check(dim, dims, h, D, reactions, caps, True, absorbing)
    assert rows > 0
