"""The C++20 facade (include/mk/markovkit.hpp): a MarkovKit-style program (tests/cpp/facade_test.cpp)
compiles against it with g++ and links the in-tree library (CPU), and runs correctly on a B200
(GPU)."""

import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "markovkit_b200"
SRC = ROOT / "tests" / "cpp" / "facade_test.cpp"
OUT = ROOT / "tests" / "cpp" / "_build" / "facade_test"


def _build() -> Path:
    if not (LIBDIR / "libmarkovkit_b200.so").exists():
        from markovkit_b200 import build

        build.build()
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", str(SRC),
           f"-L{LIBDIR}", "-lmarkovkit_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(OUT)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return OUT


def test_facade_program_compiles_and_links():
    assert _build().exists()


@pytest.mark.gpu
def test_facade_program_runs(cuda):
    exe = _build()
    proc = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600,
                          env={**os.environ, "LD_LIBRARY_PATH": str(LIBDIR)})
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "checks passed" in proc.stdout
