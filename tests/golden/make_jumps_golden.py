"""Generate tests/golden/jumps_golden.npz: the reference generator's jumps(j) for every state
(markovkit/generator.hpp:27-53 over reaction_diffusion::transitions,
markovkit/rdme/reaction_diffusion.hpp:82-118), in the reference's order, on small problems.

Runs oracle/_ref/ref_driver (MarkovKit's own headers compiled against the numerics shim by
oracle/Makefile; it needs the reference tree, so this runs only where that exists) with
dump_jumps=1 and stores per case `<case>/first` (offsets, N + 1), `<case>/to` and `<case>/rate`.

usage: python tests/golden/make_jumps_golden.py
"""

from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
DRIVER = ROOT / "oracle" / "_ref" / "ref_driver"
OUT = Path(__file__).resolve().parent / "jumps_golden.npz"

CASES = {
    # tests/test_rdme.cpp:122-140: two voxels, birth-death, cap 3
    "two_voxel_birth_death": dict(dim=1, cells=2, h=1.0, cap="3", model="birth_death", birth=2.0, death=0.25, D=0.5),
    "annihilation_2d3": dict(dim=2, cells=3, cap="1,1", model="annihilation", k=10.0, D=1.0, D2=0.5),
    "birth_death_3d2_cap2": dict(dim=3, cells=2, cap="2", model="birth_death", birth=0.05, death=0.02, D=1.5),
    "diffusion_1d5_cap3_reflecting": dict(dim=1, cells=5, cap="3", model="diffusion", D=2.0, boundary="reflecting"),
}


def main() -> None:
    arrays, meta = {}, {}
    for name, spec in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            args = [str(DRIVER)] + [f"{k}={v}" for k, v in spec.items()]
            args += ["do_apply=0", "do_mg=0", "do_plain=0", "dump_jumps=1", f"out={tmp}"]
            proc = subprocess.run(args, capture_output=True, text=True, check=True)
            m = json.loads(proc.stdout.strip().splitlines()[-1])
            for part in ("first", "to", "rate"):
                arrays[f"{name}/{part}"] = np.fromfile(Path(tmp) / f"jumps_{part}.f64", dtype=np.float64)
            meta[name] = {"spec": spec, "N": m["N"]}
            print(name, m["N"], int(arrays[f"{name}/first"][-1]), "jumps")
    arrays["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
