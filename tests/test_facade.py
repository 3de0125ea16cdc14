"""The C++20 facade (include/mk/markovkit.hpp): a MarkovKit-style program (tests/cpp/facade_test.cpp)
compiles against it with g++ and links the in-tree library (CPU), and runs correctly on a B200
(GPU). The reference's own RDME benchmark program (examples/rdme_multigrid_benchmark.cpp, which
compares plain, Jacobi, ILU(0) and multigrid-preconditioned GMRES) compiles unchanged against
the facade with -I include/mk where the reference tree is at hand (MK_REFERENCE_ROOT, else a
`reference` folder beside the repository); the binary lands in tests/cpp/_build and runs on a
B200 with --quick. The reference's own tests/test_ssa.cpp, tests/test_rdme.cpp and
tests/test_fsp.cpp build the same way and pass on the B200."""

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


REF = Path(os.environ.get("MK_REFERENCE_ROOT", ROOT.parent / "reference"))
REF_BENCH = REF / "examples" / "rdme_multigrid_benchmark.cpp"
REF_BENCH_OUT = ROOT / "tests" / "cpp" / "_build" / "rdme_multigrid_benchmark"
# the reference's own tests: SSA (gillespie, tau_leaping, trajectory, transitions) and RDME
# (voxel domains over grids and explicit graphs, population spaces, generator, population and
# sector multigrid with transfers, resolvent solves, the annihilation transform)
REF_SSA = REF / "tests" / "test_ssa.cpp"
REF_SSA_OUT = ROOT / "tests" / "cpp" / "_build" / "reference_test_ssa"
REF_RDME = REF / "tests" / "test_rdme.cpp"
REF_RDME_OUT = ROOT / "tests" / "cpp" / "_build" / "reference_test_rdme"
# FSP: distribution, expand, the generator over a listed support, adaptive and Krylov FSP
# (the latter over everywhere(), the default region)
REF_FSP = REF / "tests" / "test_fsp.cpp"
REF_FSP_OUT = ROOT / "tests" / "cpp" / "_build" / "reference_test_fsp"


def test_facade_program_compiles_and_links():
    assert _build().exists()


def test_reference_benchmark_compiles_against_facade():
    if not REF_BENCH.exists():
        pytest.skip("the reference tree is not here")
    _build()
    cmd = ["g++", "-std=c++20", "-O2", f"-I{ROOT / 'include' / 'mk'}", str(REF_BENCH), f"-L{LIBDIR}",
           "-lmarkovkit_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(REF_BENCH_OUT)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr[-4000:]
    assert REF_BENCH_OUT.exists()


@pytest.mark.parametrize("src,out", [(REF_SSA, REF_SSA_OUT), (REF_RDME, REF_RDME_OUT), (REF_FSP, REF_FSP_OUT)],
                         ids=["ssa", "rdme", "fsp"])
def test_reference_test_compiles_against_facade(src, out):
    if not src.exists():
        pytest.skip("the reference tree is not here")
    _build()
    cmd = ["g++", "-std=c++20", "-O2", f"-I{ROOT / 'include' / 'mk'}", f"-I{REF / 'tests'}", str(src),
           f"-L{LIBDIR}", "-lmarkovkit_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(out)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr[-4000:]


@pytest.mark.gpu
@pytest.mark.parametrize("out", [REF_SSA_OUT, REF_RDME_OUT, REF_FSP_OUT], ids=["ssa", "rdme", "fsp"])
def test_reference_test_runs(cuda, out):
    """the reference's tests/test_ssa.cpp, test_rdme.cpp and test_fsp.cpp, unchanged, on the device:
    every check passes (their exit status counts the failed checks)"""
    if not out.exists():
        pytest.skip("the reference test was not built against the facade")
    proc = subprocess.run([str(out)], capture_output=True, text=True, timeout=600,
                          env={**os.environ, "LD_LIBRARY_PATH": str(LIBDIR)})
    assert proc.returncode == 0, proc.stdout + proc.stderr


@pytest.mark.gpu
def test_facade_program_runs(cuda):
    exe = _build()
    proc = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600,
                          env={**os.environ, "LD_LIBRARY_PATH": str(LIBDIR)})
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "checks passed" in proc.stdout


@pytest.mark.gpu
def test_reference_benchmark_runs(cuda):
    """--quick: five small boxes, each solved plain and with the Jacobi, ILU(0) and multigrid
    preconditioners; the multigrid runs converge, every converged run reaches the same solution
    (1e-6 relative, the benchmark's own column), and the multigrid takes no more iterations than
    plain GMRES(50)."""
    if not REF_BENCH_OUT.exists():
        pytest.skip("the reference benchmark was not built against the facade")
    proc = subprocess.run([str(REF_BENCH_OUT), "--quick"], capture_output=True, text=True, timeout=600,
                          env={**os.environ, "LD_LIBRARY_PATH": str(LIBDIR)})
    assert proc.returncode == 0, proc.stdout + proc.stderr
    lines = proc.stdout.strip().splitlines()
    head = lines[0].split(",")
    rows = [dict(zip(head, ln.split(","))) for ln in lines[1:]]
    assert len(rows) == 20
    by_case = {}
    for r in rows:
        if r["method"] == "multigrid":
            assert r["converged"] == "1", r
        if r["converged"] == "1":
            assert float(r["relative_solution_difference"]) < 1e-6, r
        by_case.setdefault((r["dimension"], r["cells_per_axis"]), {})[r["method"]] = int(r["iterations"])
    for case, it in by_case.items():
        assert it["multigrid"] <= it["plain"], (case, it)
