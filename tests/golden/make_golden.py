"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs oracle/_ref/ref_driver (MarkovKit's own headers compiled against the numerics shim by
oracle/Makefile; it needs the reference tree, so this runs only where that exists) on small
seeded problems and stores its inputs and outputs as .npz. Inputs (x, b) are generated here
with markovkit_b200.inputs and handed to the driver as files, so both sides see identical
bytes.

usage: python tests/golden/make_golden.py [case ...]
"""

from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from markovkit_b200.inputs import dirichlet_rhs, uniform01, uniform_rhs  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"
OUT = Path(__file__).resolve().parent

# name -> problem (keys of ref_driver) and the right-hand side
CASES = {
    # configuration 0 of the benchmark: 1-D, 16 voxels, h = 1/16, birth-death, box cap 3
    "cfg0_birth_death_1d16": dict(dim=1, cells=16, cap="3", model="birth_death", birth=0.05, death=0.02, D=1.0, shift=0.5, rhs="uniform", seed=0, transfer=True, states=True),
    # the reference's own resolvent test problem (tests/test_rdme.cpp:225-251)
    "test_rdme_resolvent_1d4": dict(dim=1, cells=4, h=1.0, cap="3", model="birth_death", birth=0.05, death=0.02, D=4.0, shift=0.5, rhs="cos", seed=0, restart=35, maxit=200, states=True, transfer=True),
    # the reference's annihilation transform problem (tests/test_rdme.cpp:253-297)
    "annihilation_1d4": dict(dim=1, cells=4, h=0.25, cap="1,1", model="annihilation", k=2.0, D=1.0, shift=0.5, rhs="uniform", seed=5, states=True, transfer=True),
    # a small copy of configuration 1: 2-D annihilation, Dirichlet right-hand side
    "annihilation_2d8": dict(dim=2, cells=8, cap="1,1", model="annihilation", k=10.0, D=1.0, shift=1.0, rhs="dirichlet", seed=1, transfer=True),
    # a small copy of configuration 2: 3-D birth-death, box cap 2
    "birth_death_3d4_cap2": dict(dim=3, cells=4, cap="2", model="birth_death", birth=0.05, death=0.02, D=1.0, shift=0.5, rhs="uniform", seed=2, transfer=True),
    # several molecules per species with annihilation, and a reflecting boundary
    "annihilation_1d6_cap2": dict(dim=1, cells=6, cap="2,2", model="annihilation", k=3.0, D=0.5, D2=2.0, shift=0.7, rhs="uniform", seed=7, transfer=True, states=True),
    "birth_death_2d4_reflecting": dict(dim=2, cells=4, cap="2", model="birth_death", birth=0.4, death=0.3, D=2.0, shift=0.3, rhs="uniform", seed=9, boundary="reflecting", transfer=True),
    "diffusion_1d8_cap4": dict(dim=1, cells=8, cap="4", model="diffusion", D=1.5, shift=1.0, rhs="uniform", seed=11, transfer=True, states=True),
    # lists of four molecules with births and deaths (sources of the death in-jumps in every voxel)
    # an odd grid that cannot coarsen: every sector is a dense terminal block (up to 1820 states)
    "birth_death_1d13_cap4": dict(dim=1, cells=13, cap="4", model="birth_death", birth=0.6, death=0.3, D=1.2, shift=0.8, rhs="uniform", seed=13, transfer=True),
    "birth_death_1d10_cap4": dict(dim=1, cells=10, cap="4", model="birth_death", birth=0.6, death=0.3, D=1.2, shift=0.8, rhs="uniform", seed=12, transfer=True, states=True),
}


def run_case(name: str, spec: dict, work: Path) -> dict:
    dims_n = spec["cells"] ** spec["dim"]
    args = [str(DRIVER)]
    for key in ("dim", "cells", "h", "cap", "model", "birth", "death", "k", "D", "D2", "shift", "boundary", "restart", "maxit"):
        if key in spec:
            args.append(f"{key}={spec[key]}")
    # size first: a dry run that only reports N
    probe = subprocess.run(args + ["do_apply=0", "do_mg=0", f"out={work}"], capture_output=True, text=True, check=True)
    N = json.loads(probe.stdout.strip().splitlines()[-1])["N"]
    x = uniform01(spec["seed"] + 1000, N)
    if spec["rhs"] == "uniform":
        b = uniform_rhs(spec["seed"], N)
    elif spec["rhs"] == "dirichlet":
        b = dirichlet_rhs(spec["seed"], N)
    else:
        b = 1.0 + 0.1 * np.cos(np.arange(N, dtype=np.float64))
    x.tofile(work / "x_in.f64")
    b.tofile(work / "b_in.f64")
    args += [f"x_file={work / 'x_in.f64'}", f"rhs={work / 'b_in.f64'}", f"seed={spec['seed']}", f"out={work}", "do_plain=1", "tol=1e-10"]
    if spec.get("transfer"):
        args.append("do_transfer=1")
    if spec.get("states"):
        args.append("dump_states=1")
    args.append("dump_matrix=1")  # the reference's Q.matrix() and A.matrix() (Qm_*, Am_*)
    proc = subprocess.run(args, capture_output=True, text=True, check=True)
    meta = json.loads(proc.stdout.strip().splitlines()[-1])
    out = {"meta": np.array(json.dumps({"spec": spec, "ref": meta, "voxels": dims_n}))}
    for f in sorted(work.glob("*.f64")):
        if f.name in ("x_in.f64", "b_in.f64"):
            continue
        out[f.stem] = np.fromfile(f, dtype=np.float64)
    if spec.get("states"):
        S = 2 if spec["model"] == "annihilation" else 1
        out["states"] = np.fromfile(work / "states.i32", dtype=np.int32).reshape(N, dims_n * S)
    return out


def main() -> None:
    if not DRIVER.exists():
        sys.exit("oracle/_ref/ref_driver is not built (make -C oracle)")
    only = set(sys.argv[1:])  # case names to regenerate (default: all)
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as tmp:
            data = run_case(name, spec, Path(tmp))
        np.savez_compressed(OUT / f"{name}.npz", **data)
        ref = json.loads(str(data["meta"]))["ref"]
        print(f"{name}: N={ref['N']} gmres_mg={ref.get('gmres_mg', {}).get('iterations')}")


if __name__ == "__main__":
    main()
