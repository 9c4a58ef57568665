"""Factor slots backed by the CPU supernodal Cholesky of ``supernodal_cpu.cpp``.

TEST INFRASTRUCTURE ONLY -- the timed CPU baseline, never the product.  Only
``tests/``, ``__graft_entry__`` (to build it) and the CPU-baseline leg of
``bench.py`` may use it.

``SupernodalSlots`` has the interface of ``fetd_oracle.SuperLUSlots`` (the
role of ``pardiso_multi_real_mpi``, src/FETD_UTILITY.f90:826-1028), so
``fetd_oracle.run_fetd(model, slots=SupernodalSlots(model))`` runs the
oracle's adaptive BDF2 loop on a multithreaded supernodal Cholesky, as the
reference runs it on MKL PARDISO.  Dense kernels are the OpenBLAS that scipy
ships, reached through scipy's exported BLAS/LAPACK function pointers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libsupernodal_cpu.so")
SOURCES = [os.path.join(HERE, "supernodal_cpu.cpp"), os.path.join(ROOT, "temf3dt_b200", "csrc", "symbolic.cpp")]

_lib = None


def build(force: bool = False) -> str:
    """Compile the shared library next to this file (g++, OpenMP)."""
    newest = max(os.path.getmtime(s) for s in SOURCES + [os.path.join(ROOT, "temf3dt_b200", "csrc", "symbolic.h")])
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", LIB_PATH] + SOURCES
    subprocess.run(cmd, check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.sncpu_create.restype = C.c_void_p
        L.sncpu_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.sncpu_destroy.argtypes = [C.c_void_p]
        L.sncpu_factor.restype = C.c_int
        L.sncpu_factor.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.sncpu_solve.restype = C.c_int
        L.sncpu_solve.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.sncpu_release.argtypes = [C.c_void_p, C.c_int]
        L.sncpu_spmv.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _capsule_pointer(capsule) -> int:
    get_name = C.pythonapi.PyCapsule_GetName
    get_name.restype = C.c_char_p
    get_name.argtypes = [C.py_object]
    get_ptr = C.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = C.c_void_p
    get_ptr.argtypes = [C.py_object, C.c_char_p]
    return get_ptr(capsule, get_name(capsule))


class _DlInfo(C.Structure):
    _fields_ = [("dli_fname", C.c_char_p), ("dli_fbase", C.c_void_p), ("dli_sname", C.c_char_p),
                ("dli_saddr", C.c_void_p)]


def _thread_setter(any_blas_fn: int):
    """The thread-count setter of the BLAS library holding `any_blas_fn`."""
    libc = C.CDLL(None)
    info = _DlInfo()
    libc.dladdr.argtypes = [C.c_void_p, C.POINTER(_DlInfo)]
    if not libc.dladdr(C.c_void_p(any_blas_fn), C.byref(info)) or not info.dli_fname:
        return None
    blas = C.CDLL(info.dli_fname.decode())
    for name in ("scipy_openblas_set_num_threads", "openblas_set_num_threads"):
        if hasattr(blas, name):
            return C.cast(getattr(blas, name), C.c_void_p).value
    return None


def blas_table():
    """dgemm, dtrsm, dpotrf, dgemv, dtrsv and the thread setter, as addresses."""
    import scipy.linalg.cython_blas as cb
    import scipy.linalg.cython_lapack as cl
    b, lp = cb.__pyx_capi__, cl.__pyx_capi__
    fns = [_capsule_pointer(b["dgemm"]), _capsule_pointer(b["dtrsm"]), _capsule_pointer(lp["dpotrf"]),
           _capsule_pointer(b["dgemv"]), _capsule_pointer(b["dtrsv"])]
    fns.append(_thread_setter(fns[0]) or 0)
    return (C.c_void_p * 6)(*fns)


def host_threads() -> int:
    """The cores this process may run on, bounded by the container's CPU
    quota (cgroup cpu.max) and by 64, the OpenBLAS build's thread limit.
    OpenMP barriers stall badly when threads outnumber the CPUs they get."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    try:
        with open("/sys/fs/cgroup/cpu.max") as fh:
            quota, period = fh.read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(float(quota) / float(period))))
    except (OSError, ValueError):
        pass
    return max(1, min(n, 64))


class SupernodalSlots:
    """Two factor slots on the host cores (interface of SuperLUSlots)."""

    def __init__(self, model, threads: Optional[int] = None):
        from oracle.fetd_oracle import full_from_upper
        L = _load()
        self.threads = threads or host_threads()
        B, Cm = model.B.tocsr(), model.C.tocsr()
        self._keep = []
        arrs = []
        for M in (B, Cm):
            ip = np.ascontiguousarray(M.indptr, dtype=np.int64)
            ix = np.ascontiguousarray(M.indices, dtype=np.int32)
            v = np.ascontiguousarray(M.data, dtype=np.float64)
            self._keep += [ip, ix, v]
            arrs += [ip.ctypes.data, ix.ctypes.data, v.ctypes.data]
        ev = np.asarray(model.edg_vex, dtype=np.int64) - 1
        xyz = np.ascontiguousarray(0.5 * (model.nod_cor[ev[:, 0]] + model.nod_cor[ev[:, 1]]), dtype=np.float64)
        self.stats = np.zeros(4)
        self._blas = blas_table()
        self.h = L.sncpu_create(model.n, *arrs, xyz.ctypes.data, C.cast(self._blas, C.c_void_p), self.threads,
                                self.stats.ctypes.data)
        self._keep = []
        if not self.h:
            raise RuntimeError("sncpu_create failed")
        self.n = model.n
        self.B = full_from_upper(model.B).tocsr()
        self.B.sort_indices()
        self._Bp = np.ascontiguousarray(self.B.indptr, dtype=np.int32)
        self._Bi = np.ascontiguousarray(self.B.indices, dtype=np.int32)
        self._Bv = np.ascontiguousarray(self.B.data, dtype=np.float64)
        self.slot_of: Dict[int, int] = {}
        self.n_factor = 0
        self.n_solve = 0

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.sncpu_destroy(h)
            self.h = None

    def _slot(self, key: int) -> int:
        if key not in self.slot_of:
            used = set(self.slot_of.values())
            free = [s for s in (0, 1) if s not in used]
            if not free:
                raise RuntimeError("both factor slots are in use")
            self.slot_of[key] = free[0]
        return self.slot_of[key]

    def factor(self, slot: int, dt: float) -> None:
        st = _load().sncpu_factor(self.h, self._slot(slot), float(dt))
        self.n_factor += 1
        if st != 0:
            raise np.linalg.LinAlgError("supernodal Cholesky failed (status %d)" % st)

    def solve(self, slot: int, rhs: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.empty_like(b)
        if _load().sncpu_solve(self.h, self.slot_of[slot], b.ctypes.data, x.ctypes.data) != 0:
            raise RuntimeError("solve on a slot that is not factored")
        self.n_solve += 1
        return x

    def release(self, slot: int) -> None:
        s = self.slot_of.pop(slot, None)
        if s is not None:
            _load().sncpu_release(self.h, s)

    def spmv_B(self, x: np.ndarray) -> np.ndarray:
        """M_sigma x on the host threads (mkl_sparse_d_mv runs threaded)."""
        xv = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        _load().sncpu_spmv(self.h, self.n, self._Bp.ctypes.data, self._Bi.ctypes.data, self._Bv.ctypes.data,
                           xv.ctypes.data, y.ctypes.data)
        return y
