"""Generate the full-size golden solutions in tests/golden/ from the reference itself.

Runs oracle/_ref/ref_driver (MarkovKit's own headers compiled against the numerics shim by
oracle/Makefile; it needs the reference tree, so this runs only where that exists) on the
2-D 32 x 32 two-particle annihilation box of 1,050,625 states (the benchmark's second
configuration) and on the 3-D 8^3 birth-death box of cap 2 (131,841 states), and stores each
right-hand side's GMRES + sector_multigrid solution (tolerance 1e-10 relative, restart 30) as
.npz. The right-hand sides are the seeded ones of markovkit_b200.inputs, regenerated by the tests.
The 2-D case takes several minutes of single-threaded set-up in the reference.

usage: python tests/golden/make_full_golden.py [name ...]
"""

from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"
OUT = Path(__file__).resolve().parent

CASES = {
    "full_annihilation_2d32": dict(dim=2, cells=32, cap="1,1", model="annihilation", k=10.0, D=1.0,
                                   shift=1.0, rhs="dirichlet", seed=1),
    "full_birth_death_3d8_cap2": dict(dim=3, cells=8, cap="2", model="birth_death", birth=0.05,
                                      death=0.02, D=1.0, shift=0.5, rhs="uniform", seed=2),
}


def run_case(name: str, spec: dict) -> None:
    with tempfile.TemporaryDirectory() as tmp:
        args = [str(DRIVER)]
        for key in ("dim", "cells", "cap", "model", "birth", "death", "k", "D", "shift"):
            if key in spec:
                args.append(f"{key}={spec[key]}")
        args += [f"rhs={spec['rhs']}", f"seed={spec['seed']}", "tol=1e-10", "restart=30", "do_apply=0",
                 "do_plain=0", f"out={tmp}"]
        proc = subprocess.run(args, capture_output=True, text=True, check=True)
        meta = json.loads(proc.stdout.strip().splitlines()[-1])
        x = np.fromfile(Path(tmp) / "x_mg.f64", dtype=np.float64)
    np.savez_compressed(OUT / f"{name}.npz", x_mg=x,
                        meta=np.array(json.dumps({"spec": spec, "ref": meta})))
    print(name, x.size, json.dumps(meta)[:300])


def main() -> None:
    names = sys.argv[1:] or list(CASES)
    for name in names:
        run_case(name, CASES[name])


if __name__ == "__main__":
    main()
