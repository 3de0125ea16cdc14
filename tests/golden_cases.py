"""The golden fixtures of tests/golden/ (made by tests/golden/make_golden.py from the
reference) and the problem each one describes."""

from __future__ import annotations

import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


@dataclass
class Case:
    name: str
    data: dict
    spec: dict
    ref: dict

    @property
    def dim(self) -> int:
        return int(self.spec["dim"])

    @property
    def dims(self) -> list[int]:
        return [int(self.spec["cells"])] * self.dim

    @property
    def spacing(self) -> list[float]:
        h = float(self.spec.get("h", 1.0 / int(self.spec["cells"])))
        return [h] * self.dim

    @property
    def caps(self) -> list[int]:
        return [int(c) for c in str(self.spec["cap"]).split(",")]

    @property
    def diffusivities(self) -> list[float]:
        D = float(self.spec.get("D", 1.0))
        if self.spec["model"] == "annihilation":
            return [D, float(self.spec.get("D2", D))]
        return [D]

    @property
    def reactions(self):
        """(change, rate(counts, volume)) pairs restating the fixture's model family."""
        m = self.spec["model"]
        if m == "birth_death":
            b, d = float(self.spec["birth"]), float(self.spec["death"])
            return [([1], lambda n, vol, b=b: b * vol), ([-1], lambda n, vol, d=d: d * n[0])]
        if m == "annihilation":
            k = float(self.spec["k"])
            return [([-1, -1], lambda n, vol, k=k: k * n[0] * n[1] / vol)]
        return []

    @property
    def absorbing(self) -> bool:
        return self.spec.get("boundary", "absorbing") == "absorbing"

    @property
    def shift(self) -> float:
        return float(self.spec["shift"])

    @property
    def n(self) -> int:
        return int(self.ref["N"])

    def csr(self, which: str):
        """the reference's assembled matrix ("Qm": Q.matrix(), "Am": A.matrix() = shift I - Q)
        as scipy CSR"""
        import scipy.sparse as sp

        ptr = self.data[f"{which}_ptr"].astype(np.int64)
        col = self.data[f"{which}_col"].astype(np.int64)
        return sp.csr_matrix((self.data[f"{which}_val"], col, ptr), shape=(self.n, self.n))


def load(name: str) -> Case:
    raw = np.load(GOLDEN / f"{name}.npz")
    data = {k: raw[k] for k in raw.files}
    meta = json.loads(str(data.pop("meta")))
    return Case(name, data, meta["spec"], meta["ref"])


def names() -> list[str]:
    """the small resolvent fixtures of make_golden.py (fsp_*.npz hold the Krylov-FSP ones,
    full_*.npz the full-size solutions of make_full_golden.py, aggregate_golden.npz the
    aggregate-block smoother's of make_aggregate_golden.py, jumps_golden.npz the generator's
    jumps of make_jumps_golden.py)"""
    return sorted(p.stem for p in GOLDEN.glob("*.npz")
                  if not p.stem.startswith(("fsp_", "full_", "aggregate_", "jumps_")))
