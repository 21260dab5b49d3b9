"""ctypes binding of ``libmultiscat_b200.so`` (the C-ABI in include/multiscat_b200.h).

The library is built in-tree by :mod:`multiscat_b200.build`.  There is no
CPU fallback: if the library is missing or cannot be loaded every solver
entry point raises.
"""

from __future__ import annotations

import ctypes
import pathlib

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libmultiscat_b200.so"

# Every function declared in include/multiscat_b200.h (checked by the tests).
EXPORTED = (
    "msc_plan_create", "msc_plan_destroy", "msc_plan_set_potential", "msc_plan_set_system",
    "msc_solve", "msc_plan_total_rows", "msc_run_multiscat", "msc_debug_apply_coupling",
    "msc_debug_apply_block_inverse", "msc_debug_apply_operator", "msc_intensities",
    "msc_last_error", "msc_version", "msc_plan_get_info", "msc_plan_set_kernel_timing",
    "msc_plan_kernel_timing", "msc_apply_operator_noalloc", "msc_debug_apply_block_inverse_f32",
    "msc_plan_uses_tensor_cores", "msc_plan_tuning_report", "msc_plan_set_adjoint",
    "msc_plan_is_adjoint", "msc_plan_set_boundary_rhs", "msc_plan_set_adjoint_rhs",
    "msc_potential_gradient", "msc_release_cached_memory", "msc_plan_set_initial_guess",
    "msc_plan_set_systems", "msc_measure_fma_peak", "msc_debug_symmetric_eigh",
    "msc_apply_lower_block", "msc_solve_lower_block",
)

MSC_OK = 0
MSC_ERR_DIMS = 1
MSC_ERR_NOT_CONVERGED = 2
MSC_ERR_CUDA = 3
MSC_ERR_NONFINITE = 4
MSC_ERR_EIGEN = 5
MSC_ERR_ARG = 6
MSC_ERR_NOT_BUILT = 7

PRECISION_FP64 = 0
PRECISION_MIXED = 1


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("n_z", ctypes.c_int32),
        ("nkx", ctypes.c_int32),
        ("nky", ctypes.c_int32),
        ("n_systems", ctypes.c_int32),
        ("restart", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("rtol", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("inner_restart", ctypes.c_int32),
        ("inner_rtol", ctypes.c_double),
        ("max_refinements", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("precond_order", ctypes.c_int32),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32),
        ("refinements", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("fp64_fallback", ctypes.c_int32),
        ("residual", ctypes.c_double),
        ("basis_vectors", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("total_rows", ctypes.c_int64),
        ("n_taps", ctypes.c_int32),
        ("n_tiles", ctypes.c_int32),
        ("launches_last", ctypes.c_int64),
        ("cycles_last", ctypes.c_int32),
        ("fallbacks_last", ctypes.c_int32),
    ]


_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_lib = None


class NativeError(RuntimeError):
    def __init__(self, func: str, status: int, message: str):
        super().__init__(f"{func} failed with status {status}: {message}")
        self.status = status


def load() -> ctypes.CDLL:
    """Load the native library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m multiscat_b200.build` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.msc_plan_create.restype = ctypes.c_int
    lib.msc_plan_create.argtypes = [ctypes.POINTER(_vp), ctypes.POINTER(PlanDesc)]
    lib.msc_plan_destroy.restype = ctypes.c_int
    lib.msc_plan_destroy.argtypes = [_vp]
    lib.msc_plan_set_potential.restype = ctypes.c_int
    lib.msc_plan_set_potential.argtypes = [_vp, _dp, _dp]
    lib.msc_plan_set_system.restype = ctypes.c_int
    lib.msc_plan_set_system.argtypes = [_vp, ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _dp,
                                        _dp, _dp, ctypes.c_int32, _dp]
    lib.msc_plan_set_systems.restype = ctypes.c_int
    lib.msc_plan_set_systems.argtypes = [_vp, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_int64), _i32p, _i32p, _dp, _dp,
                                         _dp, _i32p, _dp]
    lib.msc_solve.restype = ctypes.c_int
    lib.msc_solve.argtypes = [_vp, _vp, _vp, ctypes.POINTER(Result), _vp]
    lib.msc_plan_total_rows.restype = ctypes.c_int64
    lib.msc_plan_total_rows.argtypes = [_vp]
    lib.msc_run_multiscat.restype = ctypes.c_int
    lib.msc_run_multiscat.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                      ctypes.POINTER(ctypes.c_int)]
    for name in ("msc_debug_apply_coupling", "msc_debug_apply_block_inverse",
                 "msc_debug_apply_operator", "msc_debug_apply_block_inverse_f32",
                 "msc_apply_lower_block", "msc_solve_lower_block"):
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = [_vp, _vp, _vp, _vp]
    lib.msc_intensities.restype = ctypes.c_int
    lib.msc_intensities.argtypes = [_vp, ctypes.c_int32, _vp, _vp, _vp]
    lib.msc_plan_get_info.restype = ctypes.c_int
    lib.msc_plan_get_info.argtypes = [_vp, ctypes.POINTER(PlanInfo)]
    lib.msc_plan_set_kernel_timing.restype = ctypes.c_int
    lib.msc_plan_set_kernel_timing.argtypes = [_vp, ctypes.c_int]
    lib.msc_plan_kernel_timing.restype = ctypes.c_int
    lib.msc_plan_kernel_timing.argtypes = [_vp, _dp, ctypes.POINTER(ctypes.c_int64)]
    lib.msc_apply_operator_noalloc.restype = ctypes.c_int
    lib.msc_apply_operator_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                               _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.msc_plan_tuning_report.restype = ctypes.c_char_p
    lib.msc_plan_tuning_report.argtypes = [_vp]
    lib.msc_plan_uses_tensor_cores.restype = ctypes.c_int
    lib.msc_plan_uses_tensor_cores.argtypes = [_vp]
    lib.msc_plan_set_adjoint.restype = ctypes.c_int
    lib.msc_plan_set_adjoint.argtypes = [_vp, ctypes.c_int32]
    lib.msc_plan_is_adjoint.restype = ctypes.c_int
    lib.msc_plan_is_adjoint.argtypes = [_vp]
    lib.msc_plan_set_boundary_rhs.restype = ctypes.c_int
    lib.msc_plan_set_boundary_rhs.argtypes = [_vp, _vp, ctypes.c_int32, _vp]
    lib.msc_plan_set_adjoint_rhs.restype = ctypes.c_int
    lib.msc_plan_set_adjoint_rhs.argtypes = [_vp, _vp, _vp, _vp, _vp]
    lib.msc_potential_gradient.restype = ctypes.c_int
    lib.msc_potential_gradient.argtypes = [_vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp]
    lib.msc_plan_set_initial_guess.restype = ctypes.c_int
    lib.msc_plan_set_initial_guess.argtypes = [_vp, _vp, ctypes.c_int32, _vp]
    lib.msc_debug_symmetric_eigh.restype = ctypes.c_int
    lib.msc_debug_symmetric_eigh.argtypes = [ctypes.c_int32, _dp, _dp, _dp]
    lib.msc_measure_fma_peak.restype = ctypes.c_int
    lib.msc_measure_fma_peak.argtypes = [ctypes.c_int32, ctypes.c_int32, _dp,
                                         ctypes.POINTER(ctypes.c_float), _vp]
    lib.msc_release_cached_memory.restype = ctypes.c_int
    lib.msc_release_cached_memory.argtypes = []
    lib.msc_last_error.restype = ctypes.c_char_p
    lib.msc_last_error.argtypes = []
    lib.msc_version.restype = ctypes.c_char_p
    lib.msc_version.argtypes = []
    _lib = lib
    return lib


def last_error() -> str:
    return load().msc_last_error().decode(errors="replace")


def check(func: str, status: int) -> None:
    if status != MSC_OK:
        raise NativeError(func, status, last_error())
