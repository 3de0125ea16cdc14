"""Krylov-FSP test problems shared by tests/golden/make_fsp_golden.py (which runs the reference
on them) and the GPU parity tests (which run the device kernel on them). Each case is a
reaction network with vectorised numpy propensities, a box, an initial state, a final time and
krylov_fsp_options; both sides see the same tabulated propensities."""

from __future__ import annotations

import numpy as np

from markovkit_b200.fsp import box, krylov_fsp_options, reaction, reaction_network
from markovkit_b200.fsp_models import birth_death, network_of, toggle  # noqa: F401
from markovkit_b200.inputs import fsp_batch_instances


def _chain3() -> reaction_network:
    # 0 -> A -> B -> C -> 0
    return reaction_network([
        reaction([1, 0, 0], lambda x: np.full(len(x), 2.0)),
        reaction([-1, 1, 0], lambda x: 1.0 * x[:, 0]),
        reaction([0, -1, 1], lambda x: 0.5 * x[:, 1]),
        reaction([0, 0, -1], lambda x: 0.3 * x[:, 2]),
    ])


def _dimers4() -> reaction_network:
    # A + B <-> C, C -> D, D -> 0, production of A and B
    return reaction_network([
        reaction([1, 0, 0, 0], lambda x: np.full(len(x), 0.5)),
        reaction([0, 1, 0, 0], lambda x: np.full(len(x), 0.4)),
        reaction([-1, -1, 1, 0], lambda x: 0.8 * x[:, 0] * x[:, 1]),
        reaction([1, 1, -1, 0], lambda x: 0.4 * x[:, 2]),
        reaction([0, 0, -1, 1], lambda x: 0.6 * x[:, 2]),
        reaction([0, 0, 0, -1], lambda x: 0.5 * x[:, 3]),
    ])


def _signed_rates() -> reaction_network:
    # rates that are zero or negative on parts of the box: those jumps do not exist
    return reaction_network([
        reaction([1], lambda x: np.where(x[:, 0] % 3 == 0, 0.0, 4.0)),
        reaction([-1], lambda x: np.where(x[:, 0] > 6, -1.0, 0.7 * x[:, 0])),
        reaction([2], lambda x: np.where(x[:, 0] < 4, 1.0, 0.0)),
    ])


def cases() -> dict:
    """name -> (network, initial, final_time, options)"""
    out = {}
    # the reference's pure-death test (tests/test_fsp.cpp:79-90); box(5) holds every state
    out["pure_death_5"] = (
        reaction_network([reaction([-1], lambda x: x[:, 0].astype(np.float64))]),
        [5], 1.0, krylov_fsp_options(inside=box([5]), tolerance=1e-10, max_steps=100, krylov_tol=1e-12))
    out["birth_death_two_layers"] = (birth_death(5.0, 0.1), [0], 0.5,
                                     krylov_fsp_options(inside=box([10]), layers=2))
    out["birth_death_small_krylov"] = (birth_death(12.0, 0.3), [3], 2.0,
                                       krylov_fsp_options(inside=box([120]), tolerance=1e-8, krylov_dim=4))
    out["birth_death_leaky_box"] = (birth_death(5.0, 0.1), [0], 2.0,
                                    krylov_fsp_options(inside=box([25]), tolerance=1e-4))
    out["birth_death_heavy_drop"] = (birth_death(8.0, 0.2), [0], 2.0,
                                     krylov_fsp_options(inside=box([200]), tolerance=1e-8,
                                                        drop_probability=1e-5, drop_derivative=1e-2))
    out["birth_death_steps"] = (birth_death(3.0, 0.5), [2], 1.5,
                                krylov_fsp_options(inside=box([60]), initial_step=0.1, step_growth=1.5))
    out["birth_death_max_steps"] = (birth_death(3.0, 0.5), [0], 5.0,
                                    krylov_fsp_options(inside=box([60]), initial_step=0.05, max_steps=12))
    out["chain3"] = (_chain3(), [0, 0, 0], 1.0, krylov_fsp_options(inside=box([8, 8, 8]), tolerance=1e-6))
    out["dimers4"] = (_dimers4(), [1, 1, 0, 0], 1.0, krylov_fsp_options(inside=box([7, 7, 5, 5]), tolerance=1e-3))
    out["signed_rates"] = (_signed_rates(), [1], 1.0, krylov_fsp_options(inside=box([12]), tolerance=1e-6))
    out["no_reactions"] = (reaction_network([]), [2, 3], 1.0, krylov_fsp_options(inside=box([4, 4])))
    out["zero_time"] = (birth_death(1.0, 1.0), [1], 0.0, krylov_fsp_options(inside=box([5])))
    inst = fsp_batch_instances()
    for k in (0, 1, 2):
        out[f"cfg_birth_death_{k}"] = (network_of(inst[k]), inst[k]["initial"], inst[k]["final_time"],
                                       krylov_fsp_options(inside=box(inst[k]["bounds"]), tolerance=inst[k]["tolerance"]))
    for k in (256, 257, 258):
        out[f"cfg_toggle_{k}"] = (network_of(inst[k]), inst[k]["initial"], inst[k]["final_time"],
                                  krylov_fsp_options(inside=box(inst[k]["bounds"]), tolerance=inst[k]["tolerance"]))
    # a toggle whose box (63 x 244) cuts through a likely region: the leak budget forces tiny
    # steps, so it stops at max_steps long before t = 2
    k = 295
    out[f"cfg_toggle_{k}_capped"] = (network_of(inst[k]), inst[k]["initial"], inst[k]["final_time"],
                                     krylov_fsp_options(inside=box(inst[k]["bounds"]), tolerance=inst[k]["tolerance"],
                                                        max_steps=300))
    return out


def table_line(path: str, initial, final_time: float, o: krylov_fsp_options) -> str:
    """the oracle driver's `table` line for a case whose propensity table is at path"""
    g = lambda v: repr(float(v))  # noqa: E731
    return " ".join([
        "table", f"path={path}", f"T={g(final_time)}", f"tol={g(o.tolerance)}", f"ktol={g(o.krylov_tol)}",
        f"kdim={o.krylov_dim}", f"layers={o.layers}", f"step={g(o.initial_step)}", f"growth={g(o.step_growth)}",
        f"drop_p={g(o.drop_probability)}", f"drop_d={g(o.drop_derivative)}", f"max_steps={int(min(o.max_steps, 2**31 - 1))}",
        "init=" + ",".join(str(int(v)) for v in initial)])
