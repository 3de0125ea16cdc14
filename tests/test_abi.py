"""Non-GPU checks of the C ABI: the in-tree library loads and exports every function that
include/*.h declares, and the ctypes signatures cover exactly those functions."""

import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "markovkit_b200" / "libmarkovkit_b200.so"


def declared() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(mk_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib_built():
    if not LIB.exists():
        from markovkit_b200 import build

        build.build()
    return LIB


def test_library_exports_every_declared_symbol(lib_built):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_built)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\b(mk_[a-z0-9_]+)\b", out))
    missing = declared() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_and_binds(lib_built):
    from markovkit_b200 import _lib

    lib = _lib.load()
    for name in declared():
        assert hasattr(lib, name)
    assert lib.mk_version() >= 1


def test_ctypes_signatures_match_header():
    from markovkit_b200 import _lib

    assert set(_lib.exported_symbols()) == declared()


def test_no_gpu_needed_for_errors(lib_built):
    """Argument errors are reported before any device work."""
    import ctypes as C

    from markovkit_b200 import _lib

    lib = _lib.load()
    out = C.c_void_p()
    rc = lib.mk_space_create_box(0, 1, (C.c_int * 1)(3), C.byref(out))
    assert rc == _lib.MK_EINVAL
    assert b"voxel" in lib.mk_last_error()


def test_server_options_are_checked_before_device_work(lib_built):
    import ctypes as C

    from markovkit_b200 import _lib

    lib = _lib.load()
    o = _lib.ServerOptions()
    lib.mk_server_options_default(C.byref(o))
    assert o.slots >= 1 and o.precision == 1 and o.rel_tolerance == 1e-10
    o.slots = 0
    h = C.c_void_p()
    assert lib.mk_server_create(C.byref(o), C.byref(h)) == _lib.MK_EINVAL
    assert b"slots" in lib.mk_last_error()


def test_matrix_and_time_step_arguments_checked_before_device_work(lib_built):
    """The assembled-generator and time-stepping entry points reject missing handles and bad
    arguments with MK_EINVAL and a message, before touching a device."""
    import ctypes as C

    from markovkit_b200 import _lib

    lib = _lib.load()
    m = C.c_void_p()
    assert lib.mk_generator_matrix(None, C.byref(m), None) == _lib.MK_EINVAL
    assert lib.mk_generator_characteristic_matrix(None, 0.5, C.byref(m), None) == _lib.MK_EINVAL
    n = C.c_int64()
    assert lib.mk_generator_n_jumps(None, C.byref(n), None) == _lib.MK_EINVAL
    rows, nnz = C.c_int64(), C.c_int64()
    assert lib.mk_csr_size(None, C.byref(rows), C.byref(nnz)) == _lib.MK_EINVAL
    lib.mk_csr_destroy(None)  # a null handle is ignored
    assert lib.mk_solver_time_steps(None, 0, 1, 1e-10, None, None, None) == _lib.MK_EINVAL
    assert b"null" in lib.mk_last_error()
