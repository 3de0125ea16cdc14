"""The matrix-free CPU port of the reference's path (oracle/_ref/mf_port, test infrastructure)
against the reference's own solutions: it is the oracle of the sizes the reference's containers
cannot hold (the 3-D 16^3 box of 8.4M states), so it is checked first on the sizes they can.

Each case solves the same seeded right-hand side as the reference did (GMRES(30) + the sector
multigrid, tolerance 1e-10 relative) and must agree with the reference's solution within 1e-8
relative, the tolerance the solutions are compared at."""

import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PORT = ROOT / "oracle" / "_ref" / "mf_port"
GOLDEN = ROOT / "tests" / "golden"

# fixture -> the port's problem keys
CASES = {
    "cfg0_birth_death_1d16": dict(dim=1, cells=16, cap="3", model="birth_death", birth=0.05, death=0.02, D=1.0,
                                  shift=0.5, rhs="uniform", seed=0),
    "full_birth_death_3d8_cap2": dict(dim=3, cells=8, cap="2", model="birth_death", birth=0.05, death=0.02,
                                      D=1.0, shift=0.5, rhs="uniform", seed=2),
    "full_annihilation_2d32": dict(dim=2, cells=32, cap="1,1", model="annihilation", k=10.0, D=1.0, shift=1.0,
                                   rhs="dirichlet", seed=1),
}


def port_solution(spec: dict) -> tuple[np.ndarray, dict]:
    with tempfile.TemporaryDirectory() as tmp:
        args = [str(PORT), *[f"{k}={v}" for k, v in spec.items()], "tol=1e-10", "restart=30",
                f"threads={os.cpu_count() or 1}", "solves=1", f"out={tmp}"]
        proc = subprocess.run(args, capture_output=True, text=True, check=True, timeout=1200)
        meta = json.loads(proc.stdout.strip().splitlines()[-1])
        return np.fromfile(Path(tmp) / "x_port.f64", dtype=np.float64), meta


@pytest.mark.skipif(not PORT.exists(), reason="oracle/_ref/mf_port is not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_reference_solution(name):
    path = GOLDEN / f"{name}.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    ref = np.load(path)["x_mg"]
    x, meta = port_solution(CASES[name])
    assert x.shape == ref.shape
    assert meta["converged"] and meta["true_rel_residual"] <= 1e-10
    rel = float(np.linalg.norm(x - ref) / np.linalg.norm(ref))
    assert rel <= 1e-8, rel
