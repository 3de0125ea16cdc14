"""The reaction networks of the batching workload, as reaction_network values for fsp.py:
birth-death ({+1} at b, {-1} at d x) and the two-species toggle switch ({+1,0} at
a1 / (1 + y^n1), {0,+1} at a2 / (1 + x^n2), unit degradation {-1,0} at x and {0,-1} at y).
The same propensities are written into the oracle's Krylov-FSP driver, so both sides tabulate
identical values."""

from __future__ import annotations

import numpy as np

from .fsp import reaction, reaction_network


def birth_death(b: float, d: float) -> reaction_network:
    return reaction_network([reaction([1], lambda x: np.full(len(x), b)),
                             reaction([-1], lambda x: d * x[:, 0])])


def toggle(a1: float, a2: float, n1: float, n2: float) -> reaction_network:
    return reaction_network([
        reaction([1, 0], lambda x: a1 / (1.0 + np.power(x[:, 1].astype(np.float64), n1))),
        reaction([0, 1], lambda x: a2 / (1.0 + np.power(x[:, 0].astype(np.float64), n2))),
        reaction([-1, 0], lambda x: x[:, 0].astype(np.float64)),
        reaction([0, -1], lambda x: x[:, 1].astype(np.float64)),
    ])


def network_of(inst: dict) -> reaction_network:
    """the network of one instance of markovkit_b200.inputs.fsp_batch_instances"""
    if inst["family"] == "birth_death":
        return birth_death(float(inst["birth"]), float(inst["death"]))
    return toggle(float(inst["a1"]), float(inst["a2"]), float(inst["n1"]), float(inst["n2"]))
