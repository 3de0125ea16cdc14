"""ctypes bindings of the C ABI in include/markovkit_b200.h.

The shared library is built in-tree (markovkit_b200/build.py). There is no fallback: if it
is missing or fails to load, every entry point raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmarkovkit_b200.so"

MK_OK = 0
MK_EINVAL = 1
MK_EOVERFLOW = 2
MK_ESINGULAR = 3
MK_ENOMEM = 4
MK_ENOTCONV = 5
MK_ENAN = 6
MK_ETIMEOUT = 7
MK_ECUDA = 8
MK_ETOLERANCE = 9
MK_ECANCELED = 10


class MkError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class InvalidArgument(MkError, ValueError):
    pass


class OverflowErrorMk(MkError, OverflowError):
    pass


_EXC = {MK_EINVAL: InvalidArgument, MK_EOVERFLOW: OverflowErrorMk}


class MultigridOptions(C.Structure):
    _fields_ = [
        ("pre_sweeps", C.c_int),
        ("post_sweeps", C.c_int),
        ("jacobi_weight", C.c_double),
        ("coarsest_size", C.c_int64),
        ("max_levels", C.c_int),
        ("coarse_cycles", C.c_int),
        ("sweep_growth", C.c_int),
        ("smoother", C.c_int),
        ("precision", C.c_int),
        ("batch", C.c_int),
        ("cycle_type", C.c_int),
    ]


class GmresOptions(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double),
        ("max_iterations", C.c_int64),
        ("restart", C.c_int),
        ("flexible", C.c_int),
    ]


class FspOptions(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double),
        ("initial_step", C.c_double),
        ("step_growth", C.c_double),
        ("drop_probability", C.c_double),
        ("drop_derivative", C.c_double),
        ("layers", C.c_int),
        ("krylov_dim", C.c_int),
        ("max_steps", C.c_int64),
        ("krylov_tol", C.c_double),
        ("method", C.c_int),
        ("step_scale", C.c_double),
        ("prune_fraction", C.c_double),
        ("flux_tolerance", C.c_double),
        ("min_probability", C.c_double),
    ]


class FspProblem(C.Structure):
    _fields_ = [
        ("n_species", C.c_int),
        ("n_reactions", C.c_int),
        ("bounds", C.POINTER(C.c_int)),
        ("change", C.POINTER(C.c_int)),
        ("rates", C.POINTER(C.c_double)),
        ("initial", C.POINTER(C.c_int)),
        ("final_time", C.c_double),
        ("options", FspOptions),
    ]


class SsaProblem(C.Structure):
    _fields_ = [
        ("n_species", C.c_int),
        ("n_reactions", C.c_int),
        ("bounds", C.POINTER(C.c_int)),
        ("change", C.POINTER(C.c_int)),
        ("rates", C.POINTER(C.c_double)),
        ("initial", C.POINTER(C.c_int)),
        ("final_time", C.c_double),
        ("method", C.c_int),
        ("max_jumps", C.c_int64),
        ("leap_step", C.c_double),
        ("leap_epsilon", C.c_double),
        ("leap_min_step", C.c_double),
        ("paths", C.c_int64),
        ("seed", C.c_uint64),
        ("n_observations", C.c_int),
        ("observation_times", C.POINTER(C.c_double)),
        ("record", C.c_int),
    ]


class SsaOutput(C.Structure):
    _fields_ = [
        ("final_state", C.POINTER(C.c_int)),
        ("observed", C.POINTER(C.c_int)),
        ("steps", C.POINTER(C.c_int64)),
        ("status", C.POINTER(C.c_int)),
        ("record_times", C.POINTER(C.c_double)),
        ("record_states", C.POINTER(C.c_int)),
        ("record_count", C.POINTER(C.c_int)),
    ]


class FspResult(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("attempts", C.c_int64),
        ("accepted", C.c_int64),
        ("support", C.c_int64),
        ("substeps", C.c_int64),
        ("applies", C.c_int64),
        ("status", C.c_int),
        ("clipped", C.c_int),
    ]


class ServerOptions(C.Structure):
    _fields_ = [
        ("slots", C.c_int),
        ("hbm_budget", C.c_size_t),
        ("precision", C.c_int),
        ("smoother", C.c_int),
        ("restart", C.c_int),
        ("max_iterations", C.c_int64),
        ("rel_tolerance", C.c_double),
        ("batch", C.c_int),
        ("coarsest_size", C.c_int64),
    ]


class ServerResult(C.Structure):
    _fields_ = [
        ("ticket", C.c_int64),
        ("status", C.c_int),
        ("iterations", C.c_int64),
        ("residual", C.c_double),
        ("latency_ms", C.c_double),
        ("queue_ms", C.c_double),
        ("solve_ms", C.c_double),
        ("batched", C.c_int),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_int64),
        ("p50_ms", C.c_double),
        ("p99_ms", C.c_double),
        ("solves_per_s", C.c_double),
        ("resident_bytes", C.c_size_t),
        ("budget_bytes", C.c_size_t),
        ("resident_solvers", C.c_int64),
        ("evictions", C.c_int64),
        ("memory_waits", C.c_int64),
    ]


class SolverResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("residual", C.c_double),
        ("converged", C.c_int),
        ("status", C.c_int),
    ]


P = C.c_void_p
I64 = C.c_int64
I64P = C.POINTER(C.c_int64)
IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)
# int (*)(void *ctx, const double *v, double *z, int64_t n)
PRECOND_HOST_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, DP, DP, C.c_int64)

# name: (restype, argtypes)
SIGNATURES = {
    "mk_last_error": (C.c_char_p, []),
    "mk_version": (C.c_int, []),
    "mk_kernel_launches": (C.c_int, [C.POINTER(C.c_uint64)]),
    "mk_set_row_path": (C.c_int, [C.c_int]),
    "mk_device_alloc": (C.c_int, [C.c_size_t, C.POINTER(P)]),
    "mk_device_free": (C.c_int, [P]),
    "mk_memcpy_h2d": (C.c_int, [P, P, C.c_size_t, P]),
    "mk_memcpy_d2h": (C.c_int, [P, P, C.c_size_t, P]),
    "mk_stream_synchronize": (C.c_int, [P]),
    "mk_space_create_box": (C.c_int, [I64, C.c_int, IP, C.POINTER(P)]),
    "mk_space_create_sector": (C.c_int, [I64, C.c_int, IP, C.POINTER(P)]),
    "mk_space_destroy": (None, [P]),
    "mk_space_size": (C.c_int, [P, I64P]),
    "mk_space_n_sectors": (C.c_int, [P, I64P]),
    "mk_space_sector_begin": (C.c_int, [P, I64, I64P]),
    "mk_space_sector_totals": (C.c_int, [P, I64, IP]),
    "mk_space_find_sector": (C.c_int, [P, IP, I64P]),
    "mk_space_sector_of": (C.c_int, [P, I64, I64P]),
    "mk_space_find_host": (C.c_int, [P, IP, I64P]),
    "mk_space_state_host": (C.c_int, [P, I64, IP]),
    "mk_space_rank": (C.c_int, [P, P, I64, P, P]),
    "mk_space_unrank": (C.c_int, [P, P, I64, P, P]),
    "mk_model_create_grid": (C.c_int, [C.c_int, I64P, DP, C.c_int, DP, C.POINTER(P)]),
    "mk_model_create_graph": (C.c_int, [I64, I64P, I64P, DP, DP, C.c_int, DP, C.POINTER(P)]),
    "mk_model_set_reactions": (C.c_int, [P, C.c_int, IP, IP, C.c_int, IP, DP]),
    "mk_model_n_voxels": (C.c_int, [P, I64P]),
    "mk_model_destroy": (None, [P]),
    "mk_generator_create": (C.c_int, [P, P, C.c_int, C.POINTER(P)]),
    "mk_generator_destroy": (None, [P]),
    "mk_generator_rows": (C.c_int, [P, I64P]),
    "mk_generator_exit_leak": (C.c_int, [P, P, P, P]),
    "mk_generator_apply": (C.c_int, [P, P, P, P]),
    "mk_generator_apply_shifted": (C.c_int, [P, C.c_double, P, P, P]),
    "mk_generator_apply_shifted_batch": (C.c_int, [P, C.c_double, P, P, I64, C.c_int, P]),
    "mk_generator_apply_f32": (C.c_int, [P, P, P, P]),
    "mk_generator_apply_shifted_f32": (C.c_int, [P, C.c_float, P, P, P]),
    "mk_generator_n_jumps": (C.c_int, [P, I64P, P]),
    "mk_generator_jumps": (C.c_int, [P, I64, I64P, DP, I64, I64P]),
    "mk_generator_matrix": (C.c_int, [P, C.POINTER(P), P]),
    "mk_generator_characteristic_matrix": (C.c_int, [P, C.c_double, C.POINTER(P), P]),
    "mk_csr_size": (C.c_int, [P, I64P, I64P]),
    "mk_csr_device": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "mk_csr_copy_host": (C.c_int, [P, I64P, I64P, C.POINTER(C.c_double)]),
    "mk_csr_destroy": (None, [P]),
    "mk_csr_create_host": (C.c_int, [I64, I64P, I64P, DP, C.POINTER(P)]),
    "mk_csr_apply": (C.c_int, [P, C.c_double, C.c_double, P, P, P]),
    "mk_multigrid_options_default": (None, [C.POINTER(MultigridOptions)]),
    "mk_multigrid_create": (C.c_int, [P, P, C.c_double, C.POINTER(MultigridOptions), C.POINTER(P)]),
    "mk_multigrid_create_full": (C.c_int, [P, C.POINTER(P), C.c_int, C.c_double, C.POINTER(MultigridOptions), C.POINTER(P)]),
    "mk_multigrid_stationary": (C.c_int, [P, P, P, P, C.c_double, I64, C.POINTER(SolverResult), P]),
    "mk_multigrid_destroy": (None, [P]),
    "mk_multigrid_apply": (C.c_int, [P, P, P, P]),
    "mk_multigrid_apply_batch": (C.c_int, [P, P, I64, P, I64, C.c_int, P]),
    "mk_multigrid_apply_noalloc": (C.c_int, [P, P, P, P]),
    "mk_multigrid_max_levels": (C.c_int, [P, IP]),
    "mk_multigrid_depth": (C.c_int, [P, IP]),
    "mk_multigrid_level_size": (C.c_int, [P, C.c_int, I64P]),
    "mk_multigrid_restrict": (C.c_int, [P, C.c_int, P, P, P]),
    "mk_multigrid_prolong": (C.c_int, [P, C.c_int, P, P, P]),
    "mk_multigrid_apply_system": (C.c_int, [P, C.c_int, P, P, P]),
    "mk_multigrid_smooth": (C.c_int, [P, C.c_int, P, P, P]),
    "mk_gmres_options_default": (None, [C.POINTER(GmresOptions)]),
    "mk_solver_create": (C.c_int, [P, C.c_double, P, C.POINTER(GmresOptions), C.POINTER(P)]),
    "mk_solver_destroy": (None, [P]),
    "mk_solver_set_tolerance": (C.c_int, [P, C.c_double]),
    "mk_solver_solve": (C.c_int, [P, P, P, C.POINTER(SolverResult), P]),
    "mk_solver_solve_host": (C.c_int, [P, P, P, C.POINTER(SolverResult), P]),
    "mk_solver_time_steps": (C.c_int, [P, C.c_int, C.c_int, C.c_double, P, C.POINTER(SolverResult), P]),
    "mk_solver_create_pc": (C.c_int, [P, C.c_double, P, C.POINTER(GmresOptions), C.POINTER(P)]),
    "mk_precond_create_diagonal": (C.c_int, [I64, DP, C.POINTER(P)]),
    "mk_precond_create_ilu0": (C.c_int, [I64, I64P, I64P, DP, P, C.POINTER(P)]),
    "mk_precond_create_multigrid": (C.c_int, [P, P, C.c_double, C.POINTER(MultigridOptions), C.POINTER(P)]),
    "mk_precond_create_host": (C.c_int, [I64, PRECOND_HOST_FN, P, C.POINTER(P)]),
    "mk_precond_destroy": (None, [P]),
    "mk_precond_size": (C.c_int, [P, I64P]),
    "mk_precond_apply": (C.c_int, [P, P, P, P]),
    "mk_precond_ilu0_schedule": (C.c_int, [P, I64P, I64P, I64P]),
    "mk_batch_solver_create": (C.c_int, [P, C.c_double, P, C.POINTER(GmresOptions), C.c_int, C.POINTER(P)]),
    "mk_batch_solver_destroy": (None, [P]),
    "mk_batch_solver_solve": (C.c_int, [P, P, P, I64, C.c_int, DP, C.POINTER(SolverResult), P]),
    "mk_fsp_options_default": (None, [C.POINTER(FspOptions)]),
    "mk_fsp_box_size": (C.c_int, [C.c_int, IP, I64P]),
    "mk_fsp_batch_create": (C.c_int, [C.c_int, C.POINTER(FspProblem), C.POINTER(P)]),
    "mk_fsp_batch_destroy": (None, [P]),
    "mk_fsp_batch_output_size": (C.c_int, [P, I64P, I64P]),
    "mk_fsp_batch_set_shape": (C.c_int, [P, C.c_int, C.c_int]),
    "mk_fsp_batch_get_shape": (C.c_int, [P, IP, IP]),
    "mk_fsp_batch_autotune": (C.c_int, [P, C.c_int, P]),
    "mk_fsp_batch_run": (C.c_int, [P, P]),
    "mk_fsp_batch_device_output": (C.c_int, [P, C.POINTER(P)]),
    "mk_fsp_batch_results": (C.c_int, [P, DP, C.POINTER(FspResult), P]),
    "mk_fsp_krylov_batch": (C.c_int, [C.c_int, C.POINTER(FspProblem), DP, C.POINTER(FspResult), P]),
    "mk_ssa_problem_default": (None, [C.POINTER(SsaProblem)]),
    "mk_ssa_run": (C.c_int, [C.POINTER(SsaProblem), C.POINTER(SsaOutput), P]),
    "mk_server_options_default": (None, [C.POINTER(ServerOptions)]),
    "mk_server_create": (C.c_int, [C.POINTER(ServerOptions), C.POINTER(P)]),
    "mk_server_destroy": (None, [P]),
    "mk_server_register": (C.c_int, [P, P, P, IP]),
    "mk_server_footprint": (C.c_int, [P, C.c_int, C.POINTER(C.c_size_t)]),
    "mk_server_submit": (C.c_int, [P, C.c_int, C.c_double, P, P, I64P]),
    "mk_server_wait": (C.c_int, [P, I64, C.POINTER(ServerResult)]),
    "mk_server_wait_for": (C.c_int, [P, I64, C.c_double, C.POINTER(ServerResult)]),
    "mk_server_cancel": (C.c_int, [P, I64]),
    "mk_server_drain": (C.c_int, [P]),
    "mk_server_stats_get": (C.c_int, [P, C.POINTER(ServerStats)]),
}

_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Load the in-tree library once and attach every declared signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise MkError(MK_ECUDA, f"{LIB_PATH.name} is not built; run markovkit_b200/build.py")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, allow: tuple[int, ...] = ()) -> int:
    if rc == MK_OK or rc in allow:
        return rc
    msg = load().mk_last_error().decode(errors="replace")
    raise _EXC.get(rc, MkError)(rc, msg)


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
