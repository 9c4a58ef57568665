"""CPU FP64 adjoint of the FETD forward run.

TEST INFRASTRUCTURE ONLY -- the checker, never the product.  Only ``tests/``
use it.  Its gradient is pinned against central finite differences of the
oracle's own forward run (``tests/test_oracle_adjoint.py``).

The reference has no readable adjoint: its inversion module ships only as
compiled objects, which are not used.  This module is the independent
restatement the GPU adjoint is checked against; it follows the mathematics.

Forward run as a graph.  With the accept/reject decisions of the adaptive
schedule held fixed (src/FETD_FWD.f90:1312-1421), every linear solve of the
run is a node

    A_k x_k = M (4 x_{a_k} - x_{b_k}) - c_k s,     A_k = 3 M + 2 dt_k K,

where a_k, b_k are the earlier nodes the BDF2 history holds at that moment
(node 0 is the initial state), M = sum_t sigma_t M_t is the sigma-mass matrix,
c_k the source scalar of sys_right (src/FETD_FWD.f90:1466-1511).  The coarse
trial solve only feeds the accept/reject test and is not a node.  Receiver
samples of an output row are linear in the node the row reports.

Adjoint.  For J(x_1..x_N), with lambda_j = 0 for j > N,

    A_k lambda_k = -dJ/dx_k + M (4 sum_{j: a_j = k} lambda_j - sum_{j: b_j = k} lambda_j),

    dJ/dsigma_t = sum_k lambda_k^T M_t (3 x_k - 4 x_{a_k} + x_{b_k}),

and dJ/dlog(sigma_c) = sum_{t in cell c} sigma_t dJ/dsigma_t.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np
import scipy.sparse.linalg as spla

from . import fetd_oracle as O


@dataclass
class Graph:
    dt: List[float] = field(default_factory=list)      # per node (index k-1 for node k)
    coef: List[float] = field(default_factory=list)    # 2 dt * pulse sign * dI/dt (0 once the source is off)
    a: List[int] = field(default_factory=list)
    b: List[int] = field(default_factory=list)
    row_node: List[int] = field(default_factory=list)  # output row -> node (row 0 -> 0)
    row_step: List[int] = field(default_factory=list)  # output row -> step number
    row_dt: List[float] = field(default_factory=list)  # output row -> dt
    decisions: List[bool] = field(default_factory=list)

    @property
    def n_nodes(self) -> int:
        return len(self.dt)


def source_vector(model: O.OracleModel) -> np.ndarray:
    """drc * edge length on the source edges (sys_right, src/FETD_FWD.f90:1507)."""
    s = np.zeros(model.n)
    for i in range(len(model.src_edg)):
        k = model.src_edg[i] - 1
        s[k] = model.src_drc[i] * model.edg_len[k]
    return s


def forward_graph(model: O.OracleModel, decisions: Optional[Sequence[bool]] = None,
                  max_steps: Optional[int] = None, legacy_linux: bool = False):
    """Replay adap_euler (pulse types 1, 2) recording the node graph.

    ``decisions`` (accept = True) replaces the error test; None uses the test.
    ``legacy_linux`` restarts BDF2 after an accepted trial from
    all_e(idx - sp_dblesize) and advances the time by one more old step (the
    build that wrote the shipped LINUX/*.field files).
    Returns (graph, states, rows) with states[k] the state of node k and rows
    the 9-component output rows as solution_output would write them.
    """
    ctl = model.ctl
    if ctl.src_pulsetype == 3:
        raise NotImplementedError("the adjoint covers runs from rest (pulse types 1 and 2)")
    slots = O.SuperLUSlots(model)
    s_vec = source_vector(model)
    n = model.n
    dbl, dsz = ctl.step_dble, ctl.step_dblesize
    g = Graph()
    states: List[np.ndarray] = [np.zeros(n)]
    out = O._Output(model)

    def coef(step_, t_, dt_):
        if step_ >= ctl.step_dvsi:
            return 0.0
        return 2.0 * dt_ * O.time_const_p(ctl.src_sourcetype, ctl.src_pulsetype, t_, ctl.src_pulsewidth,
                                          ctl.src_current)

    def node(slot, dt_, c_, a_, b_):
        rhs = slots.spmv_B(4.0 * states[a_] - states[b_]) - c_ * s_vec
        x = slots.solve(slot, rhs)
        states.append(x)
        g.dt.append(dt_); g.coef.append(c_); g.a.append(a_); g.b.append(b_)
        return len(states) - 1

    def row(step_, t_, dt_, k):
        out(step_, t_, dt_, states[k])
        g.row_node.append(k)
        g.row_step.append(step_)
        g.row_dt.append(dt_)

    step, time_cur, not_changed = 0, 0.0, 0
    step_cur = ctl.src_pulsewidth / ctl.step_dvsi
    e2 = e3 = 0
    all_e: List[int] = []
    ind, trial = 1, 0
    while time_cur < ctl.time_maxm:
        if max_steps is not None and step >= max_steps:
            break
        step += 1
        time_cur += step_cur
        if step == 1:
            row(0, time_cur - step_cur, step_cur, 0)
            slots.factor(ind, step_cur)
        if step % dbl == 0:
            t2, t3 = e2, e3
            tt = time_cur
            fine = []
            for i in range(dsz):
                k = node(ind, step_cur, coef(step, tt, step_cur), t2, t3)
                fine.append(k)
                t3, t2 = t2, k
                tt += step_cur
            tmp_step_cur = step_cur * dsz
            tmp_time_cur = time_cur - step_cur + tmp_step_cur
            other = 2 if ind == 1 else 1
            slots.factor(other, tmp_step_cur)
            rh = slots.spmv_B(4.0 * states[all_e[-1]] - states[all_e[-1 - dsz]]) \
                - coef(step, tmp_time_cur, tmp_step_cur) * s_vec
            e_veri_2 = slots.solve(other, rh)
            err = O.two_error(e_veri_2, states[fine[-1]])
            if decisions is not None:
                accept = bool(decisions[trial])
            else:
                accept = not (err > 1.0e-4 and not_changed < 2)
            trial += 1
            g.decisions.append(accept)
            if not accept:
                slots.release(other)
                row(step, time_cur, step_cur, fine[0])
                e3, e2 = e2, fine[0]
                not_changed += 1
            else:
                slots.release(ind)
                ind = other
                e3 = all_e[-1 - dsz] if legacy_linux else all_e[-1]
                e2 = fine[-1]
                time_cur = tmp_time_cur + (step_cur if legacy_linux else 0.0)
                step_cur = tmp_step_cur
                row(step, time_cur, step_cur, fine[-1])
                not_changed = 0
            all_e = []
            continue
        k = node(ind, step_cur, coef(step, time_cur, step_cur), e2, e3)
        row(step, time_cur, step_cur, k)
        all_e.append(k)
        e3, e2 = e2, k
    return g, states, np.array(out.rows)


def unit_mass_elements(model: O.OracleModel) -> np.ndarray:
    """Per-tet sigma-free mass matrices with orientation signs, (T,6,6)."""
    a, b, c, d, vol, tet_len = O.geometry(model.nod_cor, model.tet_vex)
    F = O.f_kind_iso(b, c, d, vol, tet_len, np.ones(len(vol)))
    sgn = model.tet_drc[:, :, None] * model.tet_drc[:, None, :]
    return F * sgn


def receiver_weights(model: O.OracleModel) -> np.ndarray:
    """W[r, q, j]: sample q (ex,ey,ez,dBx/dt,dBy/dt,dBz/dt) of receiver r per
    local edge j of its tet, orientation folded in (src/FETD_FWD.f90:1532-1540)."""
    R = len(model.rec_tet)
    W = np.zeros((R, 6, 6))
    for r in range(R):
        it = model.rec_tet[r] - 1
        W[r, 0:3, :] = (model.n_arr[r] * model.tet_drc[it][:, None]).T
        W[r, 3:6, :] = (model.d_arr[r] * model.tet_drc[it][:, None]).T
    return W


def adjoint_gradient(model: O.OracleModel, g: Graph, states: List[np.ndarray], dJ_dsamples: np.ndarray,
                     tet_cell: np.ndarray, ncell: int, per_tet: bool = False):
    """dJ/dlog(sigma_c) for J whose derivative with respect to the receiver
    samples (rows x nrec x 6: E and dB/dt) is dJ_dsamples.  tet_cell: cell of
    each tet (0-based), -1 outside the inversion grid.  per_tet=True also
    returns dJ/dsigma_t for every tet."""
    B = O.full_from_upper(model.B)
    C = O.full_from_upper(model.C)
    N = g.n_nodes
    W = receiver_weights(model)
    Fu = unit_mass_elements(model)
    te = model.tet_edg - 1
    # dJ/dx_k from the rows reporting node k (row 0 reports the fixed initial state)
    gx: Dict[int, np.ndarray] = {}
    for row, k in enumerate(g.row_node):
        if k == 0:
            continue
        v = gx.setdefault(k, np.zeros(model.n))
        for r in range(len(model.rec_tet)):
            edges = te[model.rec_tet[r] - 1]
            np.add.at(v, edges, W[r].T @ dJ_dsamples[row, r, :6])
    kids_a: Dict[int, List[int]] = {}
    kids_b: Dict[int, List[int]] = {}
    for j in range(1, N + 1):
        kids_a.setdefault(g.a[j - 1], []).append(j)
        kids_b.setdefault(g.b[j - 1], []).append(j)
    lam: Dict[int, np.ndarray] = {}
    G = np.zeros(len(model.tet_vex))
    fac: Dict[float, object] = {}
    for k in range(N, 0, -1):
        dt = g.dt[k - 1]
        if dt not in fac:
            fac[dt] = spla.splu((3.0 * B + 2.0 * dt * C).tocsc(), permc_spec="MMD_AT_PLUS_A",
                                diag_pivot_thresh=0.0, options={"SymmetricMode": True})
        v = np.zeros(model.n)
        for j in kids_a.get(k, []):
            v += 4.0 * lam[j]
        for j in kids_b.get(k, []):
            v -= lam[j]
        rhs = B @ v - gx.get(k, 0.0)
        lk = fac[dt].solve(rhs)
        lam[k] = lk
        w = 3.0 * states[k] - 4.0 * states[g.a[k - 1]] + states[g.b[k - 1]]
        G += np.einsum("ti,tij,tj->t", lk[te], Fu, w[te])
    grad = np.zeros(ncell)
    inside = tet_cell >= 0
    np.add.at(grad, tet_cell[inside], (model.sig * G)[inside])
    return (grad, G) if per_tet else grad


def fields_grad_to_samples(dJ_dfields: np.ndarray, steps, dts) -> np.ndarray:
    """dJ/d(receiver samples) (rows x nrec x 6) from dJ/d(output fields)
    (rows x nrec x 9).  The fields are E, dB/dt (reported 0 on step-0 rows)
    and b_i = sum_{m <= i} dB/dt_m * dt_m (solution_output,
    src/FETD_FWD.f90:1565-1620)."""
    g = np.zeros(dJ_dfields.shape[:2] + (6,))
    g[:, :, :3] = dJ_dfields[:, :, :3]
    tail = np.cumsum(dJ_dfields[::-1, :, 6:9], axis=0)[::-1]
    live = (np.asarray(steps) != 0)[:, None, None]
    g[:, :, 3:6] = live * (dJ_dfields[:, :, 3:6] + tail * np.asarray(dts)[:, None, None])
    return g


def with_sigma(model: O.OracleModel, sig: np.ndarray) -> O.OracleModel:
    """Same mesh with another conductivity per tet (re-assembles M_sigma)."""
    m = copy.copy(model)
    a, b, c, d, vol, tet_len = O.geometry(model.nod_cor, model.tet_vex)
    m.sig = sig
    m.B = O.assemble_upper(model.n, model.tet_edg, model.tet_drc, O.f_kind_iso(b, c, d, vol, tet_len, sig))
    return m
