"""Generate tests/golden/aggregate_golden.npz: the reference's sector_multigrid with
relaxation::aggregate_block (markovkit/rdme/multigrid.hpp:239-341) on small problems.

Runs oracle/_ref/ref_driver (MarkovKit's own headers compiled against the numerics shim by
oracle/Makefile; it needs the reference tree, so this runs only where that exists) with
smoother=aggregate and stores, per case, one cycle applied to the seeded right-hand side
(`<case>/Mb`) and the GMRES(30) + multigrid solution at 1e-10 (`<case>/x_mg`). The right-hand
sides are the seeded ones of markovkit_b200.inputs (regenerated by the tests).

usage: python tests/golden/make_aggregate_golden.py
"""

from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"
OUT = Path(__file__).resolve().parent / "aggregate_golden.npz"

CASES = {
    # the reference test's multigrid problem (tests/test_rdme.cpp:160-223) as a box of cap 2
    "multigrid_1d8_cap2": dict(dim=1, cells=8, h=1.0, cap="2", model="diffusion", D=1.0, shift=1.0, rhs="uniform", seed=21),
    "cfg0_birth_death_1d16": dict(dim=1, cells=16, cap="3", model="birth_death", birth=0.05, death=0.02, D=1.0, shift=0.5, rhs="uniform", seed=0),
    "annihilation_2d8": dict(dim=2, cells=8, cap="1,1", model="annihilation", k=10.0, D=1.0, shift=1.0, rhs="dirichlet", seed=1),
    "birth_death_3d4_cap2": dict(dim=3, cells=4, cap="2", model="birth_death", birth=0.05, death=0.02, D=1.0, shift=0.5, rhs="uniform", seed=2),
    "diffusion_2d4_cap3": dict(dim=2, cells=4, cap="3", model="diffusion", D=1.5, shift=0.8, rhs="uniform", seed=13),
}


def main() -> None:
    arrays, meta = {}, {}
    for name, spec in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            args = [str(DRIVER)]
            for key in ("dim", "cells", "h", "cap", "model", "birth", "death", "k", "D", "shift"):
                if key in spec:
                    args.append(f"{key}={spec[key]}")
            args += [f"rhs={spec['rhs']}", f"seed={spec['seed']}", "tol=1e-10", "restart=30", "do_apply=0",
                     "do_plain=0", "smoother=aggregate", f"out={tmp}"]
            proc = subprocess.run(args, capture_output=True, text=True, check=True)
            m = json.loads(proc.stdout.strip().splitlines()[-1])
            arrays[f"{name}/Mb"] = np.fromfile(Path(tmp) / "Mb.f64", dtype=np.float64)
            arrays[f"{name}/x_mg"] = np.fromfile(Path(tmp) / "x_mg.f64", dtype=np.float64)
            meta[name] = {"spec": spec, "ref": m}
            print(name, m["N"], m["gmres_mg"])
    arrays["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
