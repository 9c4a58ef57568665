"""Host-side mirror of TEMF3DT's forward driver over the C ABI.

``FetdGPU`` owns one library context (one GPU).  Its methods follow the
reference's phases: model_mesh/model_ctl (arrays), mesh_process (assembly),
time_solver/adap_euler (the time loop) -- see include/temf_b200.h for the
reference routine each C entry point replaces.  ``run_case`` is the
equivalent of ``./FETD -f ROOT`` for a ``.mesh``/``.cntl`` pair.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import meshio
from ._lib import (TemfError, as_f64, as_i32, dptr, fortran_f64, fortran_i32, iptr, lib)


def mesh_topology(tet_vex: np.ndarray):
    """Global edges, tet->edge map and orientation (src/FETD_FWD.f90:168-244),
    computed by the library's host helper.  Returns 1-based arrays."""
    L = lib()
    T = int(tet_vex.shape[0])
    tv = fortran_i32(tet_vex)
    ne = C.c_int(0)
    rc = L.temf_mesh_count_edges(T, iptr(tv), C.byref(ne))
    if rc:
        raise TemfError(rc, "temf_mesh_count_edges")
    ev = np.zeros(2 * ne.value, dtype=np.int32)
    te = np.zeros(6 * T, dtype=np.int32)
    td = np.zeros(6 * T, dtype=np.int32)
    rc = L.temf_mesh_topology(T, iptr(tv), ne.value, iptr(ev), iptr(te), iptr(td))
    if rc:
        raise TemfError(rc, "temf_mesh_topology")
    return ev.reshape(2, -1).T.copy(), te.reshape(6, T).T.copy(), td.reshape(6, T).T.copy()


def source_edges(edg_vex: np.ndarray, src_vex: np.ndarray):
    """Map source segments to global edges and apply the reference's
    orientation convention: +1 for every segment except the last, which is -1
    (src/FETD_FWD.f90:435-448)."""
    key = edg_vex[:, 0].astype(np.int64) * (1 << 32) + edg_vex[:, 1]
    lo = np.minimum(src_vex[:, 0], src_vex[:, 1]).astype(np.int64)
    hi = np.maximum(src_vex[:, 0], src_vex[:, 1]).astype(np.int64)
    k = lo * (1 << 32) + hi
    pos = np.searchsorted(key, k)
    if len(k) and (np.any(pos >= len(key)) or np.any(key[np.minimum(pos, len(key) - 1)] != k)):
        raise ValueError("a source segment is not an edge of the mesh")
    drc = np.ones(len(k), dtype=np.int32)
    if len(k):
        drc[-1] = -1
    return (pos + 1).astype(np.int32), drc


def pardiso_checker(symm: bool, ia, ja) -> Tuple[bool, str]:
    """Structure check of a 1-based CSR matrix (pardiso_checker,
    src/FETD_UTILITY.f90:993-1027): (valid, first violation or "")."""
    ia, ja = as_i32(ia), as_i32(ja)
    ok = np.zeros(1, dtype=np.int32)
    msg = C.create_string_buffer(256)
    rc = lib().temf_pardiso_checker(1 if symm else 0, len(ia) - 1, len(ja), iptr(ia), iptr(ja), iptr(ok), msg, 256)
    if rc != 0:
        raise TemfError(rc, "temf_pardiso_checker")
    return bool(ok[0]), msg.value.decode()


@dataclass
class RunOutput:
    steps: np.ndarray
    times: np.ndarray
    dts: np.ndarray
    fields: np.ndarray          # (rows, nrec, 9)
    trial_errors: np.ndarray
    trial_accepted: np.ndarray
    ms_factor: float
    ms_steps: float
    ms_total: float
    n_factor: int
    n_solve: int
    n_launch: int


class FetdGPU:
    """One FETD model on one GPU."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.temf_create(device, C.byref(h))
        self._h = h
        if rc:
            msg = self.last_error()
            raise TemfError(rc, msg)
        self.n_edges = 0
        self.n_tets = 0
        self.nrec = 0

    # -- plumbing -----------------------------------------------------------
    def last_error(self) -> str:
        s = self._L.temf_last_error(self._h)
        return s.decode() if s else ""

    def _ck(self, rc: int, what: str) -> int:
        if rc < 0:
            raise TemfError(rc, "%s: %s" % (what, self.last_error()))
        return rc

    def close(self) -> None:
        if self._h:
            self._L.temf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- model ----------------------------------------------------------------
    def set_mesh(self, nod_cor, tet_vex, edg_vex, tet_edg, tet_drc) -> None:
        nod = fortran_f64(nod_cor)
        tv, ev, te, td = fortran_i32(tet_vex), fortran_i32(edg_vex), fortran_i32(tet_edg), fortran_i32(tet_drc)
        self.n_tets = int(np.asarray(tet_vex).shape[0])
        self.n_edges = int(np.asarray(edg_vex).shape[0])
        self._ck(self._L.temf_set_mesh(self._h, int(np.asarray(nod_cor).shape[0]), dptr(nod), self.n_tets, iptr(tv),
                                       self.n_edges, iptr(ev), iptr(te), iptr(td)), "temf_set_mesh")

    def set_media(self, sig, mu) -> None:
        s, m = as_f64(sig), as_f64(mu)
        self._ck(self._L.temf_set_media(self._h, dptr(s), dptr(m)), "temf_set_media")

    def set_analysis_options(self, leaf_size: int = 96, amalg_level: int = 2) -> None:
        """Options of the next analyse(): nested-dissection leaf size and
        supernode amalgamation (0 none, 1 light, 2 harder: the default,
        3 hardest: up to 64 columns at 25 % explicit zeros)."""
        self._ck(self._L.temf_set_analysis_options(self._h, int(leaf_size), int(amalg_level)),
                 "temf_set_analysis_options")

    def set_media_tensor(self, sig9, mu9) -> None:
        """Anisotropic media: per tet row-major 3 x 3 conductivity and
        (absolute) permeability tensors, shape (n_tets, 9)."""
        s = as_f64(np.asarray(sig9, dtype=np.float64).reshape(-1))
        m = as_f64(np.asarray(mu9, dtype=np.float64).reshape(-1))
        self._ck(self._L.temf_set_media_tensor(self._h, dptr(s), dptr(m)), "temf_set_media_tensor")

    def set_boundary(self, bound_cond: int, face_mask=None) -> None:
        """0 = PEC, 1 = first-order absorbing boundary (face_mask: 4 bits per
        tet; None = the faces that belong to one tet)."""
        fm = None
        if face_mask is not None:
            fm = np.ascontiguousarray(face_mask, dtype=np.uint8)
        self._ck(self._L.temf_set_boundary(self._h, int(bound_cond),
                                           fm.ctypes.data_as(C.POINTER(C.c_ubyte)) if fm is not None else None),
                 "temf_set_boundary")

    def analyse(self) -> None:
        self._ck(self._L.temf_analyse(self._h), "temf_analyse")

    def assemble(self) -> None:
        self._ck(self._L.temf_assemble(self._h), "temf_assemble")

    def stats(self) -> Dict[str, float]:
        s = np.zeros(10)
        self._ck(self._L.temf_analysis_stats(self._h, dptr(s)), "temf_analysis_stats")
        keys = ["n", "nnz_A", "supernodes", "levels", "nnz_L", "stored", "flops", "update_tiles",
                "t_order", "t_symbolic"]
        return dict(zip(keys, s.tolist()))

    def get_matrix(self, which: int):
        """1-based upper CSR (ia, ja, va) of M_sigma (0) or K (1), original numbering."""
        nnz = C.c_int(0)
        self._ck(self._L.temf_get_matrix(self._h, which, C.byref(nnz), None, None, None), "temf_get_matrix")
        ia = np.zeros(self.n_edges + 1, dtype=np.int32)
        ja = np.zeros(nnz.value, dtype=np.int32)
        va = np.zeros(nnz.value)
        self._ck(self._L.temf_get_matrix(self._h, which, C.byref(nnz), iptr(ia), iptr(ja), dptr(va)), "temf_get_matrix")
        return ia, ja, va

    # -- linear algebra -------------------------------------------------------
    def factor(self, slot: int, dt: float) -> int:
        return self._ck(self._L.temf_factor(self._h, slot, float(dt)), "temf_factor")

    def solve(self, slot: int, b: np.ndarray) -> np.ndarray:
        b = np.asarray(b, dtype=np.float64)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        bb = np.ascontiguousarray(b.reshape(self.n_edges, nrhs).T)   # column-major
        x = np.zeros_like(bb)
        self._ck(self._L.temf_solve(self._h, slot, nrhs, dptr(bb), dptr(x), self.n_edges), "temf_solve")
        return x.T.reshape(b.shape)

    def release(self, slot: int) -> None:
        self._ck(self._L.temf_release(self._h, slot), "temf_release")

    def spmv(self, which: int, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        xx = np.ascontiguousarray(x.reshape(self.n_edges, nrhs).T)
        y = np.zeros_like(xx)
        self._ck(self._L.temf_spmv(self._h, which, nrhs, dptr(xx), dptr(y), self.n_edges), "temf_spmv")
        return y.T.reshape(x.shape)

    # -- sources / receivers --------------------------------------------------
    def set_sources(self, columns: Sequence[Tuple[np.ndarray, np.ndarray]], source_type: int, pulse_type: int,
                    t0: float, current: float) -> None:
        ptr = [0]
        e, d = [], []
        for edg, drc in columns:
            e.extend(np.asarray(edg).tolist())
            d.extend(np.asarray(drc).tolist())
            ptr.append(len(e))
        P, E, D = as_i32(ptr), as_i32(e if e else [0]), as_i32(d if d else [0])
        self._ck(self._L.temf_set_sources(self._h, len(columns), iptr(P), iptr(E), iptr(D), source_type, pulse_type,
                                          float(t0), float(current)), "temf_set_sources")

    def locate(self, points: np.ndarray, rec_charac: float) -> np.ndarray:
        pts = fortran_f64(points)
        out = np.zeros(len(points), dtype=np.int32)
        self._ck(self._L.temf_locate_points(self._h, len(points), dptr(pts), float(rec_charac), iptr(out)),
                 "temf_locate_points")
        return out

    def set_receivers(self, rec_tet, rec_cor, rec_rhs=None) -> None:
        rt = as_i32(rec_tet)
        rc = fortran_f64(rec_cor)
        rr = as_i32(rec_rhs) if rec_rhs is not None else None
        self.nrec = len(rt)
        self._ck(self._L.temf_set_receivers(self._h, len(rt), iptr(rt), dptr(rc), iptr(rr) if rr is not None else None),
                 "temf_set_receivers")

    def receiver_operators(self):
        n = np.zeros(self.nrec * 18)
        d = np.zeros(self.nrec * 18)
        self._ck(self._L.temf_get_receiver_operators(self._h, dptr(n), dptr(d)), "temf_get_receiver_operators")
        return n.reshape(3, 6, self.nrec).transpose(2, 1, 0), d.reshape(3, 6, self.nrec).transpose(2, 1, 0)

    # -- time loop ------------------------------------------------------------------
    def run(self, sp_division: int, sp_double: int, sp_dblesize: int, time_maximum: float,
            legacy_linux: bool = False, graphs: bool = True, forced: Optional[Sequence[int]] = None,
            max_steps: int = 0) -> RunOutput:
        flags = (1 if legacy_linux else 0) | (0 if graphs else 2)
        f = as_i32(forced) if forced is not None else None
        self._ck(self._L.temf_run(self._h, int(sp_division), int(sp_double), int(sp_dblesize), float(time_maximum),
                                  flags, iptr(f) if f is not None else None, len(f) if f is not None else 0,
                                  int(max_steps)), "temf_run")
        return self.result()

    def set_mesh_fields(self, times) -> None:
        """Whole-mesh field snapshots (vtkout) for the next run; [] turns them off."""
        t = as_f64(times if len(times) else [0.0])
        self._ck(self._L.temf_set_mesh_fields(self._h, len(times), dptr(t)), "temf_set_mesh_fields")

    def mesh_fields(self, index: int):
        """(fields (n_tets, 9) = E, D, B at the snapshot, reached?) of the last run."""
        out = np.zeros(9 * self.n_tets)
        done = C.c_int(0)
        self._ck(self._L.temf_result_mesh_fields(self._h, int(index), dptr(out), C.byref(done)),
                 "temf_result_mesh_fields")
        return out.reshape(self.n_tets, 9), bool(done.value)

    def result(self) -> RunOutput:
        """Output of the last run of this context (temf_run or a batch run)."""
        rows = C.c_int(0)
        self._ck(self._L.temf_result_rows(self._h, C.byref(rows)), "temf_result_rows")
        R = rows.value
        steps = np.zeros(R, dtype=np.int32)
        times = np.zeros(R)
        dts = np.zeros(R)
        fields = np.zeros(R * max(self.nrec, 1) * 9)
        self._ck(self._L.temf_result_get(self._h, iptr(steps), dptr(times), dptr(dts), dptr(fields)),
                 "temf_result_get")
        nt = C.c_int(0)
        self._ck(self._L.temf_result_trials(self._h, C.byref(nt), None, None), "temf_result_trials")
        errs = np.zeros(max(nt.value, 1))
        acc = np.zeros(max(nt.value, 1), dtype=np.int32)
        self._ck(self._L.temf_result_trials(self._h, C.byref(nt), dptr(errs), iptr(acc)), "temf_result_trials")
        t = [C.c_double(0), C.c_double(0), C.c_double(0)]
        nf, ns, nl = C.c_int(0), C.c_int(0), C.c_longlong(0)
        self._ck(self._L.temf_result_timing(self._h, C.byref(t[0]), C.byref(t[1]), C.byref(t[2]), C.byref(nf),
                                            C.byref(ns), C.byref(nl)), "temf_result_timing")
        return RunOutput(steps, times, dts, fields.reshape(R, max(self.nrec, 1), 9), errs[:nt.value],
                         acc[:nt.value].astype(bool), t[0].value, t[1].value, t[2].value, nf.value, ns.value,
                         int(nl.value))

    def gates(self, gate_times: Sequence[float]):
        g = as_f64(gate_times)
        out = np.zeros(len(g) * max(self.nrec, 1) * 9)
        done = np.zeros(len(g), dtype=np.int32)
        self._ck(self._L.temf_result_gates(self._h, len(g), dptr(g), dptr(out), iptr(done)), "temf_result_gates")
        return out.reshape(len(g), max(self.nrec, 1), 9), done.astype(bool)

    def tune_solve(self, slot: int, nrhs: int = 1):
        """Autotune the sweeps' queue split level on the factor in `slot`;
        returns (chosen level, {level: ms per solve})."""
        sp, n = C.c_int(0), C.c_int(0)
        cs = np.zeros(8, dtype=np.int32)
        cm = np.zeros(8)
        self._ck(self._L.temf_tune_solve(self._h, slot, nrhs, C.byref(sp), C.byref(n), iptr(cs), dptr(cm)),
                 "temf_tune_solve")
        return sp.value, {int(cs[i]): float(cm[i]) for i in range(n.value)}

    def solve_schedule(self, nrhs: int = 1):
        """(split level in use, tuned?) of the single-column or block sweeps."""
        sp, tu = C.c_int(0), C.c_int(0)
        self._ck(self._L.temf_solve_schedule(self._h, nrhs, C.byref(sp), C.byref(tu)), "temf_solve_schedule")
        return sp.value, bool(tu.value)

    def set_solve_plan(self, tree_level: int, split: int, run_leaders: bool = True) -> None:
        """Single-column sweep plan: subtree level (0 = no subtrees), queue
        split level, and whether runs of column blocks above the split are
        swept by one leader task."""
        self._ck(self._L.temf_set_solve_plan(self._h, int(tree_level), int(split), 1 if run_leaders else 0),
                 "temf_set_solve_plan")

    def set_wait_limit(self, spins: int = 0, inject_unmet_wait: bool = False) -> None:
        """Polls a device wait may spin before it gives up (0: the default);
        inject_unmet_wait: the next single-column solve waits once on a count
        nothing completes (tests the timeout path)."""
        self._ck(self._L.temf_set_wait_limit(self._h, int(spins), 1 if inject_unmet_wait else 0),
                 "temf_set_wait_limit")

    def solve_plan(self) -> Dict[str, int]:
        """The single-column sweep plan in use: subtree level, queue split, run leaders, subtrees, tuned."""
        lv, sp, ld, nt, tu = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        self._ck(self._L.temf_solve_plan(self._h, C.byref(lv), C.byref(sp), C.byref(ld), C.byref(nt),
                                         C.byref(tu)), "temf_solve_plan")
        return {"tree_level": lv.value, "split": sp.value, "run_leaders": bool(ld.value), "n_trees": nt.value,
                "tuned": bool(tu.value)}

    def solve_timeline(self, slot: int):
        """Per-task timeline of one single-column solve (profiling aid):
        (forward, backward) arrays of rows (start_ns, ready_ns, end_ns, sm,
        supernode, kind, r0, level)."""
        nf, nb = C.c_int(0), C.c_int(0)
        self._ck(self._L.temf_solve_timeline(self._h, slot, 0, None, C.byref(nf), C.byref(nb)), "temf_solve_timeline")
        out = np.zeros(8 * (nf.value + nb.value), dtype=np.uint64)
        self._ck(self._L.temf_solve_timeline(self._h, slot, out.size, out.ctypes.data_as(C.POINTER(C.c_ulonglong)),
                                             C.byref(nf), C.byref(nb)), "temf_solve_timeline")
        out = out.reshape(-1, 8).astype(np.int64)
        return out[:nf.value], out[nf.value:]

    # -- adjoint gradient ---------------------------------------------------------------
    def adjoint_record(self, checkpoint_every: int = 50) -> None:
        """Record the next runs' solve graph for :meth:`adjoint` (0 = off)."""
        self._ck(self._L.temf_adjoint_record(self._h, int(checkpoint_every)), "temf_adjoint_record")

    def adjoint(self, dJ_dfields: np.ndarray, tet_cell: Optional[np.ndarray] = None, ncell: int = 0):
        """Gradient of a misfit J of the last recorded run's output.

        dJ_dfields: (rows, nrec, 9) = dJ/d(fields of :meth:`run`).  tet_cell:
        0-based inversion cell per tet, -1 outside (None: no cells).  Returns
        (dJ/dlog sigma per cell, dJ/dsigma per tet, timing dict).
        """
        g = as_f64(np.asarray(dJ_dfields, dtype=np.float64).reshape(-1))
        grad_t = np.zeros(self.n_tets)
        grad_c = np.zeros(max(int(ncell), 1))
        cell = None
        if tet_cell is not None:
            cell = as_i32(np.asarray(tet_cell, dtype=np.int64) + 1)
        self._ck(self._L.temf_adjoint(self._h, dptr(g), int(ncell), iptr(cell) if cell is not None else None,
                                      dptr(grad_c) if cell is not None else None, dptr(grad_t)), "temf_adjoint")
        ms = np.zeros(2)
        cnt = (C.c_longlong * 4)()
        self._ck(self._L.temf_adjoint_timing(self._h, dptr(ms), cnt), "temf_adjoint_timing")
        timing = dict(ms_total=float(ms[0]), ms_factor=float(ms[1]), nodes=int(cnt[0]), blocks=int(cnt[1]),
                      factors=int(cnt[2]), launches=int(cnt[3]))
        return grad_c[:int(ncell)], grad_t, timing

    # -- PARDISO-compatible shim ------------------------------------------------------
    def pardiso_alloc(self, max_matrix: int) -> None:
        self._ck(self._L.temf_pardiso_alloc(self._h, max_matrix), "temf_pardiso_alloc")

    def pardiso_direct_1(self, num_m: int, ia, ja, va) -> int:
        ia, ja, va = as_i32(ia), as_i32(ja), as_f64(va)
        return self._ck(self._L.temf_pardiso_direct_1(self._h, num_m, 1, len(ia) - 1, len(ja), iptr(ia), iptr(ja),
                                                      dptr(va)), "temf_pardiso_direct_1")

    def pardiso_direct_2(self, num_m: int, b: np.ndarray) -> np.ndarray:
        b = as_f64(b)
        x = np.zeros_like(b)
        self._ck(self._L.temf_pardiso_direct_2(self._h, num_m, dptr(b), dptr(x)), "temf_pardiso_direct_2")
        return x

    def pardiso_direct_3(self, num_m: int) -> None:
        self._ck(self._L.temf_pardiso_direct_3(self._h, num_m), "temf_pardiso_direct_3")

    def pardiso_dealloc(self) -> None:
        self._ck(self._L.temf_pardiso_dealloc(self._h), "temf_pardiso_dealloc")


class FetdBatch:
    """Several prepared models stepped together on one GPU (temf_batch_*):
    one merged forward and one merged backward solve kernel per step."""

    def __init__(self, models: Sequence[FetdGPU]):
        self._L = lib()
        self.models = list(models)
        arr = (C.c_void_p * len(self.models))(*[m._h for m in self.models])
        h = C.c_void_p()
        rc = self._L.temf_batch_create(arr, len(self.models), C.byref(h))
        self._h = h
        if rc < 0:
            msg = self._L.temf_batch_last_error(h).decode()
            self.close()
            raise TemfError(rc, "temf_batch_create: " + msg)

    def _ck(self, rc: int, what: str) -> int:
        if rc < 0:
            raise TemfError(rc, "%s: %s" % (what, self._L.temf_batch_last_error(self._h).decode()))
        return rc

    def close(self) -> None:
        if self._h:
            self._L.temf_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, sp_division: int, sp_double: int, sp_dblesize: int, time_maximum: float,
            legacy_linux: bool = False, graphs: bool = True, autotune: bool = False, max_steps: int = 0):
        flags = (1 if legacy_linux else 0) | (0 if graphs else 2) | (4 if autotune else 0)
        self._ck(self._L.temf_batch_run(self._h, int(sp_division), int(sp_double), int(sp_dblesize),
                                        float(time_maximum), flags, int(max_steps)), "temf_batch_run")
        return [m.result() for m in self.models]

    def timing(self) -> Dict[str, float]:
        ms = np.zeros(4)
        cnt = (C.c_longlong * 3)()
        self._ck(self._L.temf_batch_timing(self._h, dptr(ms), cnt), "temf_batch_timing")
        return dict(ms_total=float(ms[0]), ms_factor=float(ms[1]), ms_steps=float(ms[2]), ms_tune=float(ms[3]),
                    steps=int(cnt[0]), launches=int(cnt[1]), merged_solves=int(cnt[2]))

    def tuning(self):
        o, g = C.c_int(0), C.c_int(0)
        cand = np.zeros(6)
        tuned = self._ck(self._L.temf_batch_tuning(self._h, C.byref(o), C.byref(g), dptr(cand)), "temf_batch_tuning")
        return dict(tuned=bool(tuned), order=o.value, grid_pct=g.value, candidate_ms=cand.tolist())

    def set_tuning(self, order: int, grid_pct: int) -> None:
        self._ck(self._L.temf_batch_set_tuning(self._h, int(order), int(grid_pct)), "temf_batch_set_tuning")


def load_case(gpu: FetdGPU, mesh: meshio.Mesh, ctl: meshio.Control, rec_tet: Optional[np.ndarray] = None):
    """model_mesh + model_ctl + mesh_process for one ``.mesh``/``.cntl`` pair."""
    edg_vex, tet_edg, tet_drc = mesh_topology(mesh.tet_vex)
    gpu.set_mesh(mesh.nod_cor, mesh.tet_vex, edg_vex, tet_edg, tet_drc)
    if ctl.aniso_domains:
        sig, mu = meshio.media_tensors_per_tet(mesh.tet_phy, ctl)
        gpu.set_media_tensor(sig, mu)
    else:
        sig, mu = meshio.media_per_tet(mesh.tet_phy, ctl)
        gpu.set_media(sig, mu)
    gpu.set_boundary(ctl.bound_cond)
    gpu.analyse()
    gpu.assemble()
    src_edg, src_drc = source_edges(edg_vex, mesh.src_vex)
    gpu.set_sources([(src_edg, src_drc)], ctl.source_type, ctl.pulse_type, ctl.t0, ctl.current)
    if rec_tet is None:
        rec_tet = gpu.locate(ctl.rec_cor, ctl.rec_charac)
        if (rec_tet == 0).any():
            raise ValueError("no rec tet No. %d" % (int(np.argmin(rec_tet)) + 1))
    gpu.set_receivers(rec_tet, ctl.rec_cor)
    return dict(edg_vex=edg_vex, tet_edg=tet_edg, tet_drc=tet_drc, sig=sig, mu=mu, src_edg=src_edg,
                src_drc=src_drc, rec_tet=np.asarray(rec_tet))


def run_case(root: str, device: int = 0, legacy_linux: bool = False, write: bool = True) -> RunOutput:
    """``./FETD -f ROOT``: read ROOT.mesh/.cntl, run on the GPU, write ROOT.field(2)."""
    mesh = meshio.read_mesh(root + ".mesh")
    ctl = meshio.read_cntl(root + ".cntl")
    with FetdGPU(device) as gpu:
        load_case(gpu, mesh, ctl)
        out = gpu.run(ctl.sp_division, ctl.sp_double, ctl.sp_dblesize, ctl.time_maximum,
                      legacy_linux=legacy_linux)
        if write:
            meshio.write_field(root + ".field", out.steps, out.times, out.fields, ctl.output)
            if ctl.time_points is not None:
                g, done = gpu.gates(ctl.time_points)
                idx = np.nonzero(done)[0]
                meshio.write_field(root + ".field2", idx + 1, ctl.time_points[idx], g[idx], ctl.output)
        return out


class CaseFile:
    """ROOT.mesh + ROOT.cntl read by the library's C++ front end
    (temf_case_read: model_mesh and model_ctl); the arrays in the reference's
    conventions (1-based vertices), plus loading a context and writing the
    .field files the way the reference's driver does."""

    def __init__(self, root: str):
        L = lib()
        h = C.c_void_p()
        msg = C.create_string_buffer(512)
        rc = L.temf_case_read(root.encode(), C.byref(h), msg, 512)
        if rc != 0:
            raise ValueError(msg.value.decode() or "temf_case_read failed")
        self._L, self._h = L, h
        sz = np.zeros(7, dtype=np.int32)
        L.temf_case_sizes(h, iptr(sz))
        N, T, S, R = int(sz[0]), int(sz[1]), int(sz[2]), int(sz[3])
        nod = np.zeros(3 * N)
        tv = np.zeros(4 * T, dtype=np.int32)
        tp = np.zeros(max(T, 1), dtype=np.int32)
        sv = np.zeros(max(2 * S, 1), dtype=np.int32)
        spn = np.zeros(max(S, 1), dtype=np.int32)
        L.temf_case_mesh(h, dptr(nod), iptr(tv), iptr(tp), iptr(sv), iptr(spn))
        self.nod_cor = nod.reshape(3, N).T.copy()
        self.tet_vex = tv.reshape(4, T).T.copy()
        self.tet_phy = tp[:T].copy()
        self.src_vex = sv[:2 * S].reshape(2, S).T.copy()
        self.src_phy = spn[:S].copy()
        ints = np.zeros(10, dtype=np.int32)
        reals = np.zeros(4)
        rc_ = np.zeros(max(3 * R, 1))
        ntp = int(sz[6])
        tpts = np.zeros(max(ntp, 1))
        L.temf_case_control(h, iptr(ints), dptr(reals), dptr(rc_), dptr(tpts))
        (self.bound_cond, self.src_num, self.source_type, self.pulse_type, self.sp_mthd, self.sp_division,
         self.sp_double, self.sp_dblesize, self.vtkout) = [int(v) for v in ints[:9]]
        self.output = np.array([(int(ints[9]) >> k) & 1 == 1 for k in range(9)])
        self.rec_charac, self.t0, self.current, self.time_maximum = [float(v) for v in reals]
        self.rec_cor = rc_[:3 * R].reshape(3, R).T.copy()
        self.time_points = tpts[:ntp].copy() if ntp >= 0 else None
        self.n_iso, self.n_aniso = int(sz[4]), int(sz[5])
        nv = C.c_int(0)
        L.temf_case_vtk_times(h, C.byref(nv), None)
        vt = np.zeros(max(nv.value, 1))
        L.temf_case_vtk_times(h, C.byref(nv), dptr(vt))
        self.vtk_times = vt[:nv.value].copy()

    def close(self) -> None:
        if self._h:
            self._L.temf_case_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def media(self):
        """(sig, mu, aniso): per tet (n_tets,) or row-major tensors (n_tets, 9)."""
        T = self.tet_vex.shape[0]
        a = C.c_int(0)
        self._L.temf_case_media(self._h, None, None, C.byref(a))
        k = 9 if a.value else 1
        sig, mu = np.zeros(k * T), np.zeros(k * T)
        rc = self._L.temf_case_media(self._h, dptr(sig), dptr(mu), C.byref(a))
        if rc != 0:
            raise ValueError("error - physical domain not found!")
        return (sig.reshape(T, 9), mu.reshape(T, 9), True) if a.value else (sig, mu, False)

    def load(self, gpu: "FetdGPU") -> None:
        msg = C.create_string_buffer(512)
        if self._L.temf_case_load(self._h, gpu._h, msg, 512) != 0:
            raise ValueError(msg.value.decode())
        self.n_edges = gpu.n_edges = self._edges(gpu)
        gpu.n_tets = self.tet_vex.shape[0]
        gpu.nrec = self.rec_cor.shape[0]

    def _edges(self, gpu) -> int:
        s = np.zeros(10)
        gpu._ck(self._L.temf_analysis_stats(gpu._h, dptr(s)), "temf_analysis_stats")
        return int(s[0])

    def write_msh(self, src_msh: str, dst_msh: str, fields: np.ndarray) -> None:
        """msh_output: a copy of src_msh with $ElementData blocks of the
        selected output columns of fields (n_tets, 9) = E, D, B."""
        f = as_f64(np.asarray(fields, dtype=np.float64).reshape(-1, 9))
        msg = C.create_string_buffer(512)
        if self._L.temf_case_write_msh(self._h, src_msh.encode(), dst_msh.encode(), dptr(f), msg, 512) != 0:
            raise ValueError(msg.value.decode())

    def write(self, gpu: "FetdGPU", root: str) -> None:
        msg = C.create_string_buffer(512)
        if self._L.temf_case_write(self._h, gpu._h, root.encode(), msg, 512) != 0:
            raise RuntimeError(msg.value.decode())


def mesh_fields_host(nod_cor, tet_vex, tet_edg, tet_drc, e) -> np.ndarray:
    """vtk_field_save's E and D of the edge vector e at every tet centroid,
    (n_tets, 6) = Ex Ey Ez Dx Dy Dz (the library's host evaluation of the
    per-tet formula its GPU kernels share)."""
    nod = fortran_f64(nod_cor)
    tv, te, td = fortran_i32(tet_vex), fortran_i32(tet_edg), fortran_i32(tet_drc)
    ev = as_f64(e)
    T = int(np.asarray(tet_vex).shape[0])
    out = np.zeros(6 * T)
    rc = lib().temf_mesh_fields_host(int(np.asarray(nod_cor).shape[0]), dptr(nod), T, iptr(tv), iptr(te), iptr(td),
                                     len(ev), dptr(ev), dptr(out))
    if rc != 0:
        raise TemfError(rc, "temf_mesh_fields_host")
    return out.reshape(T, 6)


def run_case_native(root: str, device: int = 0, legacy_linux: bool = False) -> None:
    """``./FETD -f ROOT`` entirely in the library (temf_case_run)."""
    msg = C.create_string_buffer(512)
    if lib().temf_case_run(root.encode(), device, 1 if legacy_linux else 0, msg, 512) != 0:
        raise RuntimeError(msg.value.decode())


def write_field_rows(path: str, steps, times, fields: np.ndarray, output_mask) -> None:
    """The library's .field writer (temf_case_write_rows); fields (rows, nrec, 9)."""
    st = as_i32(steps)
    tm = as_f64(times)
    f = as_f64(np.asarray(fields, dtype=np.float64).reshape(len(st), -1, 9))
    m = as_i32(np.asarray(output_mask, dtype=bool).astype(np.int32))
    rc = lib().temf_case_write_rows(path.encode(), len(st), f.shape[1], iptr(st), dptr(tm), dptr(f), iptr(m))
    if rc != 0:
        raise TemfError(rc, "temf_case_write_rows")
