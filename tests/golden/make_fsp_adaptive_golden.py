"""Generate tests/golden/fsp_adaptive_golden.npz: the reference's own solve_adaptive_fsp
(markovkit/fsp.hpp:123-188) on birth-death and toggle-switch networks.

Runs oracle/_ref/ref_fsp (MarkovKit's headers compiled against the numerics shim; it needs the
reference tree, so this runs only where that exists) with adaptive=1 and stores each case's
final time and distribution. CASES lists (network line of ref_fsp, adaptive options); the GPU
test rebuilds the same networks with markovkit_b200.fsp_models.

usage: python tests/golden/make_fsp_adaptive_golden.py
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
from markovkit_b200.inputs import fsp_batch_instances  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "ref_fsp"
OUT = Path(__file__).resolve().parent / "fsp_adaptive_golden.npz"


def cases() -> dict:
    """name -> dict(family, params, bounds, initial, T, options); options use the names of
    adaptive_fsp_options"""
    inst = fsp_batch_instances()
    out = {
        # the reference's adaptive test (tests/test_fsp.cpp:68-77)
        "test_fsp_birth_death": dict(family="birth_death", birth=5.0, death=0.1, bounds=[100], initial=[0], T=2.0,
                                     options=dict(step_scale=0.1)),
        "birth_death_defaults": dict(family="birth_death", birth=12.0, death=0.3, bounds=[300], initial=[3], T=3.0,
                                     options={}),
        "birth_death_min_probability": dict(family="birth_death", birth=20.0, death=0.5, bounds=[200], initial=[0],
                                            T=1.5, options=dict(min_probability=1e-8, prune_fraction=0.3)),
        "birth_death_max_steps": dict(family="birth_death", birth=8.0, death=0.2, bounds=[150], initial=[0], T=5.0,
                                      options=dict(step_scale=0.05, max_steps=5)),
    }
    for k, opts in ((256, dict(step_scale=0.5)), (257, dict(layers=2, prune_fraction=0.2, flux_tolerance=1e-5))):
        x = inst[k]
        out[f"toggle_{k}"] = dict(family="toggle", a1=x["a1"], a2=x["a2"], n1=x["n1"], n2=x["n2"], bounds=x["bounds"],
                                  initial=x["initial"], T=2.0, options=opts)
    return out


def line(c: dict) -> str:
    g = lambda v: repr(float(v))  # noqa: E731
    o = c["options"]
    tail = ["adaptive=1", f"scale={g(o.get('step_scale', 1.0))}", f"prune={g(o.get('prune_fraction', 0.1))}",
            f"flux={g(o.get('flux_tolerance', 1e-6))}", f"minp={g(o.get('min_probability', 0.0))}",
            f"layers={int(o.get('layers', 1))}", f"max_steps={int(o.get('max_steps', 1 << 28))}"]
    if c["family"] == "birth_death":
        head = ["birth_death", g(c["birth"]), g(c["death"]), str(c["bounds"][0]), g(c["T"]), "1e-6", "1e-8", "30",
                str(c["initial"][0])]
    else:
        head = ["toggle", g(c["a1"]), g(c["a2"]), g(c["n1"]), g(c["n2"]), str(c["bounds"][0]), str(c["bounds"][1]),
                g(c["T"]), "1e-6", "1e-8", "30", str(c["initial"][0]), str(c["initial"][1])]
    return " ".join(head + tail)


def main() -> None:
    all_cases = cases()
    names = list(all_cases)
    arrays, meta = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        (tmp / "cases.txt").write_text("\n".join(line(all_cases[n]) for n in names) + "\n")
        out_dir = tmp / "out"
        out_dir.mkdir()
        proc = subprocess.run([str(DRIVER), f"file={tmp / 'cases.txt'}", f"out={out_dir}"],
                              capture_output=True, text=True, check=True)
        reports = [json.loads(r) for r in proc.stdout.strip().splitlines()]
        for k, name in enumerate(names):
            raw = np.fromfile(out_dir / f"fsp{k}.bin", dtype=np.uint8)
            pairs = raw.view(np.dtype([("i", "<i8"), ("p", "<f8")]))
            arrays[f"{name}/index"] = pairs["i"].copy()
            arrays[f"{name}/p"] = pairs["p"].copy()
            meta[name] = {"case": all_cases[name], "t": reports[k]["t"], "support": reports[k]["support"]}
            print(name, reports[k])
    arrays["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
