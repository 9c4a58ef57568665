"""ctypes binding of libtemf_b200.so (the C ABI in include/temf_b200.h).

The library is loaded from this package directory.  There is no fallback:
if the shared library is missing the import of the compute path fails with a
clear message (build it with ``python -m temf3dt_b200.build``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtemf_b200.so")

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "temf_create": (_i, [_i, C.POINTER(_p)]),
    "temf_destroy": (_i, [_p]),
    "temf_last_error": (C.c_char_p, [_p]),
    "temf_version": (C.c_char_p, []),
    "temf_mesh_count_edges": (_i, [_i, _ip, _ip]),
    "temf_mesh_topology": (_i, [_i, _ip, _i, _ip, _ip, _ip]),
    "temf_set_mesh": (_i, [_p, _i, _dp, _i, _ip, _i, _ip, _ip, _ip]),
    "temf_set_media": (_i, [_p, _dp, _dp]),
    "temf_analyse": (_i, [_p]),
    "temf_assemble": (_i, [_p]),
    "temf_get_matrix": (_i, [_p, _i, _ip, _ip, _ip, _dp]),
    "temf_factor": (_i, [_p, _i, _d]),
    "temf_solve": (_i, [_p, _i, _i, _dp, _dp, _i]),
    "temf_release": (_i, [_p, _i]),
    "temf_solve_noalloc": (_i, [_p, _i, _p, _p]),
    "temf_spmv": (_i, [_p, _i, _i, _dp, _dp, _i]),
    "temf_set_sources": (_i, [_p, _i, _ip, _ip, _ip, _i, _i, _d, _d]),
    "temf_set_receivers": (_i, [_p, _i, _ip, _dp, _ip]),
    "temf_get_receiver_operators": (_i, [_p, _dp, _dp]),
    "temf_locate_points": (_i, [_p, _i, _dp, _d, _ip]),
    "temf_run": (_i, [_p, _i, _i, _i, _d, _i, _ip, _i, _i]),
    "temf_result_rows": (_i, [_p, _ip]),
    "temf_result_get": (_i, [_p, _ip, _dp, _dp, _dp]),
    "temf_result_trials": (_i, [_p, _ip, _dp, _ip]),
    "temf_result_gates": (_i, [_p, _i, _dp, _dp, _ip]),
    "temf_result_timing": (_i, [_p, _dp, _dp, _dp, _ip, _ip, C.POINTER(C.c_longlong)]),
    "temf_analysis_stats": (_i, [_p, _dp]),
    "temf_symbolic_host": (_i, [_i, C.POINTER(C.c_longlong), _ip, _dp, _ip, _dp]),
    "temf_adjoint_record": (_i, [_p, _i]),
    "temf_set_media_tensor": (_i, [_p, _dp, _dp]),
    "temf_set_boundary": (_i, [_p, _i, C.POINTER(C.c_ubyte)]),
    "temf_set_analysis_options": (_i, [_p, _i, _i]),
    "temf_tune_solve": (_i, [_p, _i, _i, _ip, _ip, _ip, _dp]),
    "temf_solve_schedule": (_i, [_p, _i, _ip, _ip]),
    "temf_set_solve_plan": (_i, [_p, _i, _i, _i]),
    "temf_solve_plan": (_i, [_p, _ip, _ip, _ip, _ip, _ip]),
    "temf_set_wait_limit": (_i, [_p, _i, _i]),
    "temf_schedule_check": (_i, [_i, C.POINTER(C.c_longlong), _ip, _dp, C.c_char_p, _i]),
    "temf_solve_timeline": (_i, [_p, _i, C.c_longlong, C.POINTER(C.c_ulonglong), _ip, _ip]),
    "temf_batch_create": (_i, [C.POINTER(C.c_void_p), _i, C.POINTER(C.c_void_p)]),
    "temf_batch_destroy": (_i, [_p]),
    "temf_batch_last_error": (C.c_char_p, [_p]),
    "temf_batch_run": (_i, [_p, _i, _i, _i, _d, _i, _i]),
    "temf_batch_timing": (_i, [_p, _dp, C.POINTER(C.c_longlong)]),
    "temf_batch_tuning": (_i, [_p, _ip, _ip, _dp]),
    "temf_batch_set_tuning": (_i, [_p, _i, _i]),
    "temf_adjoint": (_i, [_p, _dp, _i, _ip, _dp, _dp]),
    "temf_adjoint_timing": (_i, [_p, _dp, C.POINTER(C.c_longlong)]),
    "temf_pardiso_checker": (_i, [_i, _i, _i, _ip, _ip, _ip, C.c_char_p, _i]),
    "temf_case_read": (_i, [C.c_char_p, C.POINTER(_p), C.c_char_p, _i]),
    "temf_case_free": (_i, [_p]),
    "temf_case_sizes": (_i, [_p, _ip]),
    "temf_case_mesh": (_i, [_p, _dp, _ip, _ip, _ip, _ip]),
    "temf_case_control": (_i, [_p, _ip, _dp, _dp, _dp]),
    "temf_case_media": (_i, [_p, _dp, _dp, _ip]),
    "temf_case_write_rows": (_i, [C.c_char_p, _i, _i, _ip, _dp, _dp, _ip]),
    "temf_case_vtk_times": (_i, [_p, _ip, _dp]),
    "temf_set_mesh_fields": (_i, [_p, _i, _dp]),
    "temf_result_mesh_fields": (_i, [_p, _i, _dp, _ip]),
    "temf_mesh_fields_host": (_i, [_i, _dp, _i, _ip, _ip, _ip, _i, _dp, _dp]),
    "temf_case_write_msh": (_i, [_p, C.c_char_p, C.c_char_p, _dp, C.c_char_p, _i]),
    "temf_case_load": (_i, [_p, _p, C.c_char_p, _i]),
    "temf_case_write": (_i, [_p, _p, C.c_char_p, C.c_char_p, _i]),
    "temf_case_run": (_i, [C.c_char_p, _i, _i, C.c_char_p, _i]),
    "temf_pardiso_alloc": (_i, [_p, _i]),
    "temf_pardiso_direct_1": (_i, [_p, _i, _i, _i, _i, _ip, _ip, _dp]),
    "temf_pardiso_direct_2": (_i, [_p, _i, _dp, _dp]),
    "temf_pardiso_direct_3": (_i, [_p, _i]),
    "temf_pardiso_dealloc": (_i, [_p]),
}

_lib = None


def lib():
    """Load (once) and return the shared library with typed entry points."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libtemf_b200.so not found at %s -- build it with "
                              "`python -m temf3dt_b200.build` (no CPU fallback exists)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip) if a is not None else None


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp) if a is not None else None


def as_i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)


def as_f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.float64)


def fortran_i32(a) -> np.ndarray:
    """(rows, cols) array -> column-major int32 buffer (Fortran layout)."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).T)


def fortran_f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)


class TemfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("temf error %d: %s" % (code, msg))
        self.code = code
