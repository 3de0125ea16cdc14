"""Build libmarkovkit_b200.so in-tree: every CUDA source for sm_100a, compiled in parallel.

The library is plain CUDA C++ behind a C ABI (include/markovkit_b200.h); nothing links
against torch. Objects go to markovkit_b200/_build/, the shared library next to this file.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libmarkovkit_b200.so"

PLAIN = ["row_kernels.cu", "transfer.cu", "aggregate.cu", "krylov.cu", "engine.cu", "capi.cu", "noalloc.cu", "fsp.cu",
         "capi_fsp.cu", "server.cpp", "assemble.cu", "precond.cu", "capi_precond.cu", "dense_inverse.cu",
         "ssa.cu", "capi_ssa.cu", "csr_apply.cu"]
PRECISIONS = {"f64": "double", "f32": "float"}
N_SHAPES = 10  # the state shapes of with_shape (generator_row.cuh)


def units() -> list[tuple[str, list[str], str]]:
    """(source, defines, object stem): the plain sources once each; the general row kernel once
    per (precision, batch width, state shape) and the stencil row kernel once per (precision,
    batch width), so the heavy template instantiations compile in parallel."""
    out = [(name, [], Path(name).stem) for name in PLAIN]
    for tag, t in PRECISIONS.items():
        for nb in (1, 4):
            out.append(("stencil_rows.cu", [f"-DMK_T={t}", f"-DMK_NB={nb}"], f"stencil_rows_{tag}_nb{nb}"))
            for shape in range(N_SHAPES):
                out.append(("row_kernels_inst.cu", [f"-DMK_T={t}", f"-DMK_NB={nb}", f"-DMK_SHAPE={shape}"],
                            f"row_kernels_{tag}_nb{nb}_s{shape}"))
    return out
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-std=c++20",
    "-O3",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I",
    str(ROOT / "include"),
]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return found


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{proc.stderr}")
    return obj, proc.stderr


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _local_includes(src: Path, seen: set[Path] | None = None) -> set[Path]:
    """The project headers a source includes, transitively (quoted includes found next to the
    including file or under include/)."""
    seen = set() if seen is None else seen
    for name in _INCLUDE.findall(src.read_text()):
        for base in (src.parent, ROOT / "include"):
            h = (base / name).resolve()
            if h.exists():
                if h not in seen:
                    seen.add(h)
                    _local_includes(h, seen)
                break
    return seen


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    extra = extra or []
    BUILD.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for name, defines, stem in units():
        src = CSRC / name
        obj = BUILD / (stem + ".o")
        objs.append(str(obj))
        if _stale(obj, [src, *sorted(_local_includes(src)), Path(__file__)]):
            jobs.append((src, obj, defines))
    # the slowest units first, so the pool's tail is short
    jobs.sort(key=lambda j: 0 if "row_kernels_inst" in j[0].name else 1)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            for obj, log in ex.map(lambda j: _compile(j[0], j[1], [*j[2], *extra]), jobs):
                if verbose and log.strip():
                    print(log, file=sys.stderr)
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed:\n{proc.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
