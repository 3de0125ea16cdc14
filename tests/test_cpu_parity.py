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
