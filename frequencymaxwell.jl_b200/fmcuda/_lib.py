"""ctypes binding of libfmcuda (declarations in include/fmcuda.h).

The shared library is built in-tree next to this file (see ``build.py``).  There
is no CPU fallback: importing the solver without the library, or calling it on a
machine without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os
import warnings

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfmcuda.so")

FM_OK, FM_ERR_INVALID, FM_ERR_OOM, FM_NOT_CONVERGED, FM_ERR_NONFINITE, FM_ERR_TIMEOUT, FM_ERR_CUDA, \
    FM_ERR_UNSUPPORTED = range(8)
FM_PREC_F64, FM_PREC_F32, FM_PREC_F32_MATH64 = 0, 1, 2
FM_METHOD_GMRES, FM_METHOD_BICGSTAB, FM_METHOD_RICHARDSON = 0, 1, 2
FM_ORTHO_MGS, FM_ORTHO_CGS, FM_ORTHO_CGS2, FM_ORTHO_BLOCK = 0, 1, 2, 3
FM_BLOCK_FP64, FM_BLOCK_STORAGE, FM_BLOCK_FP64_ORTHO = 0, 1, 2
FM_TUNE_Y_TMA, FM_TUNE_Z_TMA, FM_TUNE_TMA_CTAS_PER_SM, FM_TUNE_ROW_THREADS, FM_TUNE_WAVE_RHS = 0, 1, 2, 3, 4
FM_TUNE_BLOCK_DOT = 5
FM_SHAPE_SPHERE, FM_SHAPE_PLATE, FM_SHAPE_CYLINDER = 0, 1, 2

STATUS_NAMES = {
    FM_OK: "FM_OK", FM_ERR_INVALID: "FM_ERR_INVALID", FM_ERR_OOM: "FM_ERR_OOM",
    FM_NOT_CONVERGED: "FM_NOT_CONVERGED", FM_ERR_NONFINITE: "FM_ERR_NONFINITE",
    FM_ERR_TIMEOUT: "FM_ERR_TIMEOUT", FM_ERR_CUDA: "FM_ERR_CUDA", FM_ERR_UNSUPPORTED: "FM_ERR_UNSUPPORTED",
}

# Every symbol the header declares; tests check the library exports all of them.
EXPORTED = (
    "fm_abi_version", "fm_last_error", "fm_device_count", "fm_plan_create", "fm_plan_destroy", "fm_plan_bytes",
    "fm_set_potential", "fm_green_apply", "fm_apply_operator", "fm_apply_preconditioner", "fm_curl_field",
    "fm_solve_source", "fm_build_potential", "fm_solve_plane_waves", "fm_copy_fields", "fm_synchronize",
    "fm_set_profiling", "fm_kernel_stats", "fm_launch_count", "fm_stream", "fm_green_apply_noalloc",
    "fm_engine_slot_bytes", "fm_engine_slot_bytes_ortho", "fm_engine_create", "fm_engine_destroy", "fm_engine_submit", "fm_engine_step",
    "fm_engine_status", "fm_plan_set_tuning", "fm_plan_get_tuning", "fm_phantom_fill",
)


class fm_plan_desc(C.Structure):
    _fields_ = [("grid", C.c_int * 3), ("pad", C.c_int * 3), ("resolution", C.c_double * 3),
                ("absorbing", C.c_int * 3), ("precision", C.c_int), ("max_rhs", C.c_int), ("device", C.c_int)]


class fm_solve_opts(C.Structure):
    _fields_ = [("method", C.c_int), ("ortho", C.c_int), ("restart", C.c_int), ("maxiters", C.c_int),
                ("reltol", C.c_double), ("abstol", C.c_double), ("timeout_s", C.c_double), ("block", C.c_int),
                ("block_store", C.c_int)]


class fm_solve_info(C.Structure):
    _fields_ = [("iterations", C.c_int), ("solved", C.c_int), ("residual", C.c_double),
                ("residual0", C.c_double)]


class fm_potential_info(C.Structure):
    _fields_ = [("eps_imag", C.c_double), ("k_bg", C.c_double), ("bornmax", C.c_int)]


class fm_plane_wave(C.Structure):
    _fields_ = [("wavelength", C.c_double), ("polarization", C.c_double * 6), ("k_vector", C.c_double * 3),
                ("amplitude", C.c_double), ("phase", C.c_double)]


class fm_shape(C.Structure):
    _fields_ = [("kind", C.c_int), ("axis", C.c_int), ("center", C.c_double * 3), ("radius", C.c_double),
                ("extent", C.c_double), ("value", C.c_double * 2)]


class fm_kernel_stat(C.Structure):
    _fields_ = [("name", C.c_char * 16), ("launches", C.c_longlong), ("ms", C.c_double), ("bytes", C.c_double)]


class FMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """Load libfmcuda.so once; raise loudly if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libfmcuda.so not found at {LIB_PATH}; build it with "
                          f"`python -c 'import __graft_entry__ as g; g.build()'` or `make -C csrc`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    L.fm_abi_version.restype = C.c_int
    L.fm_last_error.restype = C.c_char_p
    L.fm_device_count.restype = C.c_int
    L.fm_plan_create.argtypes = [C.POINTER(fm_plan_desc), C.POINTER(P)]
    L.fm_plan_destroy.argtypes = [P]
    L.fm_plan_destroy.restype = None
    L.fm_plan_bytes.argtypes = [C.POINTER(fm_plan_desc), C.c_int, C.c_int]
    L.fm_plan_bytes.restype = C.c_longlong
    L.fm_set_potential.argtypes = [P, P, C.c_double, C.c_double, C.c_double]
    L.fm_green_apply.argtypes = [P, C.c_int, P, P]
    L.fm_apply_operator.argtypes = [P, C.c_int, P, P, C.c_double, C.c_double, C.c_double, C.c_double]
    L.fm_apply_preconditioner.argtypes = [P, C.c_int, P, P]
    L.fm_curl_field.argtypes = [P, C.c_int, P, P]
    L.fm_solve_source.argtypes = [P, C.c_int, P, C.POINTER(fm_solve_opts), P, P, C.POINTER(fm_solve_info)]
    L.fm_build_potential.argtypes = [P, P, C.c_double, C.c_double, P, P, P, C.c_int, C.POINTER(fm_potential_info)]
    L.fm_solve_plane_waves.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(fm_plane_wave), C.c_double,
                                       C.POINTER(fm_solve_opts), P, P, C.POINTER(fm_solve_info)]
    L.fm_copy_fields.argtypes = [P, C.c_int, P, P]
    L.fm_synchronize.argtypes = [P]
    L.fm_set_profiling.argtypes = [P, C.c_int]
    L.fm_kernel_stats.argtypes = [P, C.POINTER(fm_kernel_stat), C.c_int]
    L.fm_kernel_stats.restype = C.c_int
    L.fm_launch_count.argtypes = [P]
    L.fm_launch_count.restype = C.c_longlong
    L.fm_plan_set_tuning.argtypes = [P, C.c_int, C.c_int]
    L.fm_plan_set_tuning.restype = C.c_int
    L.fm_plan_get_tuning.argtypes = [P, C.c_int, C.POINTER(C.c_int)]
    L.fm_plan_get_tuning.restype = C.c_int
    L.fm_engine_slot_bytes.argtypes = [C.POINTER(fm_plan_desc), C.c_int]
    L.fm_engine_slot_bytes.restype = C.c_longlong
    L.fm_engine_slot_bytes_ortho.argtypes = [C.POINTER(fm_plan_desc), C.c_int, C.c_int]
    L.fm_engine_slot_bytes_ortho.restype = C.c_longlong
    L.fm_engine_create.argtypes = [P, C.c_int, C.c_int, C.c_double, C.c_double, P, P, P, C.c_int, C.POINTER(P)]
    L.fm_engine_create.restype = C.c_int
    L.fm_engine_destroy.argtypes = [P]
    L.fm_engine_destroy.restype = None
    L.fm_engine_submit.argtypes = [P, C.c_longlong, P, C.c_int, C.POINTER(fm_plane_wave), C.c_double, C.c_int, P, P]
    L.fm_engine_submit.restype = C.c_int
    L.fm_engine_step.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                 C.POINTER(fm_solve_info), C.c_int]
    L.fm_engine_step.restype = C.c_int
    L.fm_engine_status.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.fm_engine_status.restype = C.c_int
    L.fm_green_apply_noalloc.argtypes = [C.POINTER(fm_plan_desc), C.c_double, C.c_double, C.c_int, P, P, P]
    L.fm_green_apply_noalloc.restype = C.c_int
    L.fm_phantom_fill.argtypes = [P, C.c_double, C.c_int, C.POINTER(fm_shape), P]
    L.fm_phantom_fill.restype = C.c_int
    L.fm_stream.argtypes = [P]
    L.fm_stream.restype = C.c_void_p
    for name in ("fm_plan_create", "fm_set_potential", "fm_green_apply", "fm_apply_operator",
                 "fm_apply_preconditioner", "fm_curl_field", "fm_solve_source", "fm_build_potential",
                 "fm_solve_plane_waves", "fm_copy_fields", "fm_synchronize", "fm_set_profiling"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(status: int, allow_not_converged: bool = False) -> int:
    """Raise FMError for a failing status; FM_NOT_CONVERGED passes when allowed (the reference warns)."""
    if status == FM_OK:
        return status
    if status == FM_NOT_CONVERGED and allow_not_converged:
        return status
    msg = lib().fm_last_error().decode(errors="replace")
    if status == FM_ERR_INVALID:
        raise ValueError(msg)
    raise FMError(status, msg)


def ptr(a) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def warn_not_converged():
    # convergent_born.jl:753-755
    warnings.warn("LinearSolve.jl did not converge.", RuntimeWarning, stacklevel=3)
