"""Generate tests/golden/fsp_batch_golden.npz: instances of the Krylov-FSP batching workload
(markovkit_b200.inputs.fsp_batch_instances: 512 propagations to t = 2, tolerance 1e-8) run
through the reference's own solve_krylov_fsp (oracle/_ref/ref_fsp: MarkovKit's headers compiled
against the numerics shim; it needs the reference tree, so this runs only where that exists),
with the attempt cap the batch uses (max_steps = 2000).

The instances: the first 16 of each family, and toggles whose box cuts through a likely region
so that the leak budget forces tiny steps and they stop at the cap before t = 2.

usage: python tests/golden/make_fsp_batch_golden.py
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
from markovkit_b200.inputs import fsp_batch_instances, fsp_instance_line  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "ref_fsp"
OUT = Path(__file__).resolve().parent / "fsp_batch_golden.npz"
MAX_STEPS = 2000
CAPPED = [295]  # toggles that stop at the attempt cap (the batch records which do)
INDICES = list(range(16)) + list(range(256, 272)) + CAPPED


def main() -> None:
    inst = fsp_batch_instances()
    arrays, meta = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        (tmp / "cases.txt").write_text(
            "\n".join(fsp_instance_line(inst[k], max_steps=MAX_STEPS) for k in INDICES) + "\n")
        out_dir = tmp / "out"
        out_dir.mkdir()
        proc = subprocess.run([str(DRIVER), f"file={tmp / 'cases.txt'}", f"out={out_dir}"],
                              capture_output=True, text=True, check=True)
        reports = [json.loads(line) for line in proc.stdout.strip().splitlines()]
        for j, k in enumerate(INDICES):
            raw = np.fromfile(out_dir / f"fsp{j}.bin", dtype=np.uint8)
            pairs = raw.view(np.dtype([("i", "<i8"), ("p", "<f8")]))
            arrays[f"{k}/index"] = pairs["i"].copy()
            arrays[f"{k}/p"] = pairs["p"].copy()
            meta[str(k)] = {"t": reports[j]["t"], "support": reports[j]["support"]}
            print(k, meta[str(k)], f"{reports[j]['ms']:.1f} ms")
    arrays["meta"] = np.array(json.dumps({"max_steps": MAX_STEPS, "instances": meta}))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
