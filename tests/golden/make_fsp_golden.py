"""Generate tests/golden/fsp_cases.npz from the reference's own Krylov FSP.

Tabulates each problem of tests/fsp_cases.py over its box with markovkit_b200.fsp.tabulate,
writes the table in the `table` format of oracle/ref_fsp.cpp (MarkovKit's solve_krylov_fsp,
markovkit/fsp.hpp:207-254, compiled against the numerics shim by oracle/Makefile; it needs the
reference tree, so this runs only where that exists), runs it, and stores for every case the
final time, the number of saved snapshots and the final distribution as (box index,
probability) pairs.

usage: python tests/golden/make_fsp_golden.py
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
sys.path.insert(0, str(ROOT / "tests"))
from fsp_cases import cases, table_line  # noqa: E402

from markovkit_b200.fsp import tabulate  # noqa: E402

DRIVER = ROOT / "oracle" / "_ref" / "ref_fsp"
OUT = Path(__file__).resolve().parent / "fsp_cases.npz"


def write_table(path: Path, network, region) -> None:
    change, rates = tabulate(network, region)
    S = len(region.bounds)
    R = change.shape[0]
    with open(path, "wb") as f:
        f.write(np.array([S, R], dtype=np.int32).tobytes())
        f.write(np.asarray(region.bounds, dtype=np.int32).tobytes())
        f.write(change.astype(np.int32).tobytes())
        f.write(rates.astype(np.float64).tobytes())


def main() -> None:
    all_cases = cases()
    arrays = {}
    meta = {}
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        lines = []
        names = list(all_cases)
        for k, name in enumerate(names):
            network, initial, T, opt = all_cases[name]
            table = tmp / f"table{k}.bin"
            write_table(table, network, opt.inside)
            lines.append(table_line(str(table), initial, T, opt))
        (tmp / "cases.txt").write_text("\n".join(lines) + "\n")
        out_dir = tmp / "out"
        out_dir.mkdir()
        proc = subprocess.run([str(DRIVER), f"file={tmp / 'cases.txt'}", f"out={out_dir}"],
                              capture_output=True, text=True, check=True)
        reports = [json.loads(line) for line in proc.stdout.strip().splitlines()]
        for k, name in enumerate(names):
            raw = np.fromfile(out_dir / f"fsp{k}.bin", dtype=np.uint8)
            pairs = raw.view(np.dtype([("i", "<i8"), ("p", "<f8")]))
            arrays[f"{name}/index"] = pairs["i"].copy()
            arrays[f"{name}/p"] = pairs["p"].copy()
            meta[name] = {"t": reports[k]["t"], "support": reports[k]["support"],
                          "saved": reports[k]["saved"]}
            print(name, meta[name], f"{reports[k]['ms']:.1f} ms")
    arrays["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
