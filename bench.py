"""Benchmark: FETD time steps x RHS per second on one B200 (or N replicas).

One bench step = one complete forward FETD run of the configured model: the
adaptive BDF2 time loop from t = 0 to time_maximum with every refactorisation
at the dt-doubling trials (adap_euler, src/FETD_FWD.f90:1229-1464), i.e. the
whole job, with the mesh analysed and the matrices assembled beforehand.
  value = (time steps of the run x RHS columns x ranks) / device time of the run.
The default workload (config 1) is the 3-D block model: 0.01 S/m host,
0.1 S/m block of 200 x 200 x 100 m with its top at 100 m, air 1e-12 S/m,
1000 m square loop, 64 receivers on a 20 m line; 1 238 964 tets and
1 477 597 edges, synthetic and seeded.  Its factors (GBs) exceed the 126 MB
L2 many times over, so no L2 flush is needed between steps.

Beside the headline, on one GPU, the default line carries the other configs
of the metric:
  batched: config 2, the 64 small loops (50 x 50 m, 8 x 8 at 40 m) on the same
           mesh as one 64-column block per step, the full run, against the
           headline (plain single-RHS on the same mesh), with the dB/dt error
           of four columns against plain runs replaying the same decisions;
  models:  16 layered models of uneven size in one batch against one after another;
  adjoint: config 3, the gradient of a dB/dt misfit (64 receivers x 40 gates)
           with respect to log sigma of 32 x 32 x 16 log-normal cells on the
           same mesh, against one forward run of that model.

e2e: the same metric through the public API with host buffers: per step the
conductivity/permeability per tet and the source/receiver arrays are copied
host->device, the matrices re-assembled, the loop run and the receiver
traces copied back.

--impl reference: the reference's CPU path is Intel Fortran + MKL PARDISO,
which cannot be built or run here; its CPU restatement is timed instead: the
oracle's adaptive BDF2 loop on a multithreaded supernodal Cholesky
(oracle/supernodal_cpu.cpp, the same ordering as the GPU path, OpenMP +
OpenBLAS on all host cores), on the full-resolution model; each bench step
runs the first 10 time steps from rest, with the factorisation timed once
and amortised over a doubling period.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# The block models share one grid (the lines of the 1000 m loop and of the 8 x 8
# small loops; 44 m cells in the core, 22 m vertically near the surface):
# 1 238 964 tets, 1 477 597 edges.  Config 2 is the config-1 mesh with other
# sources and receivers; config 3 the config-1 mesh with per-cell conductivity.
BLOCK_GRID = dict(shared_grid=True, h_core=44.0, h_z=22.0)
CONFIGS = {
    0: dict(kind="halfspace", kw=dict(h_core=125, ratio=2.0, h_z=25), label="halfspace-0.001Spm-loop500m-150k-edges"),
    1: dict(kind="block", kw=dict(BLOCK_GRID), label="block3d-0.01/0.1Spm-square1000m-64rec-1.24M-tets-1.48M-edges"),
    2: dict(kind="multiloop", kw=dict(BLOCK_GRID), label="block3d-1.48M-edges-64-loops-64rhs"),
    3: dict(kind="block", kw=dict(BLOCK_GRID),
            label="block3d-1.48M-edges-lognormal-32x32x16-cells-64rec-40gates-adjoint"),
    4: dict(kind="ellipsoids", kw=dict(h_core=20.0, h_z=12.0, ratio=1.4),
            label="ellipsoids-0.005Spm-4.37M-tets-5.17M-edges-256-loops-64rhs-blocks"),
}
# config 3: the inversion grid (32 x 32 x 16 cells of 25 x 25 x 12.5 m under the
# loop), log-normal cell conductivities around 0.01 S/m with 0.5 decades, and
# the observations of a seeded perturbation of that model (0.1 decades)
INV_SHAPE = (32, 32, 16)
INV_BOX = ((-400.0, 400.0), (-400.0, 400.0), (0.0, 200.0))
GATES = np.logspace(-6, -2, 40)
COMMON = dict(t0=1e-6, sp_division=10, sp_double=100, time_maximum=1e-2)


def model_for(cfg: int, reduced: bool = False):
    from temf3dt_b200 import synth
    c = CONFIGS[cfg]
    kw = dict(c["kw"])
    kw.update(COMMON)
    if reduced:
        kw.update(dict(h_core=kw.get("h_core", 40.0) * 8, h_z=kw.get("h_z", 20.0) * 6, ratio=2.5))
    return synth.build_model(c["kind"], seed=cfg, **kw)


class Clocks:
    """Sample SM clocks and throttle reasons with nvidia-smi during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 3 + k and "Active" in r[3 + k]
                          and r[3 + k].strip() != "Not Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_dgemm_tflops(torch) -> float:
    """cuBLAS FP64 GEMM rate on this GPU (roofline denominator for the factor)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def host_cores() -> int:
    """Host threads the CPU arm may use (the process's CPUs, bounded by the
    container's CPU quota, at most 64)."""
    from oracle.supernodal_cpu import host_threads
    return host_threads()


def cpu_arm(cfg: int, steps: int, warmup: int, sample_steps: int = 0):
    """The reference's CPU path restated (oracle/): the adaptive BDF2 loop of
    fetd_oracle on the CPU supernodal Cholesky (oracle/supernodal_cpu.cpp,
    OpenMP + OpenBLAS, all host cores), on the full-resolution model of the
    config.  One bench step = the loop's first `sample_steps` time steps from
    rest (default 10: BDF2 right-hand side, source, solve, receivers), on the
    factor of the first dt.  That factorisation is timed once, at warm-up,
    and amortised over one doubling period, as the full run has about one
    factorisation per sp_double steps (10 in 995 on the block model):
        steps/s = 1 / (seconds per time step + factorisation s / sp_double).
    Falls back to the reduced-resolution model when a factor slot does not
    fit in free host memory."""
    from oracle import fetd_oracle as O
    from oracle import supernodal_cpu as SN
    from tests.golden_cases import synth_oracle_model
    threads = host_cores()
    SN.build()
    reduced = False
    om = synth_oracle_model(model_for(cfg))
    slots = SN.SupernodalSlots(om, threads=threads)
    try:
        import psutil
        if 8 * slots.stats[2] + 4e9 > psutil.virtual_memory().available:
            del slots
            reduced = True
            om = synth_oracle_model(model_for(cfg, reduced=True))
            slots = SN.SupernodalSlots(om, threads=threads)
    except ImportError:
        pass
    period = int(om.ctl.step_dble)
    S = sample_steps or 10
    dt0 = om.ctl.src_pulsewidth / om.ctl.step_dvsi
    # the factor of the first dt is computed once and reused by every sample
    t0 = time.perf_counter()
    slots.factor(1, dt0)
    fac_s = time.perf_counter() - t0
    factor, release = slots.factor, slots.release
    held = {1: dt0}

    def cached_factor(slot, dt):
        if held.get(slot) != dt:
            factor(slot, dt)
            held[slot] = dt

    def keep_release(slot):
        if slot != 1:
            release(slot)
            held.pop(slot, None)

    slots.factor, slots.release = cached_factor, keep_release
    rhs = np.ones(om.n)
    for _ in range(warmup):   # one solve per warm-up step
        slots.solve(1, rhs)
    vals, secs = [], []
    for _ in range(steps):
        t = time.perf_counter()
        res = O.run_fetd(om, max_steps=S, slots=slots)
        dt = time.perf_counter() - t
        n = len(res.steps) - 1
        vals.append(1.0 / (dt / n + fac_s / period))
        secs.append(dt)
    info = dict(n_edges=om.n, steps=S, seconds=float(np.mean(secs)), threads=threads, reduced=reduced,
                factor_s=fac_s, stored=float(slots.stats[2]))
    how = ("%d time steps from rest per sample (%.1f s), on the factor of the first dt; its factorisation "
           "(%.1f s, timed once) amortised over one doubling period (%d steps)" % (S, info["seconds"], fac_s, period))
    text = ("CPU restatement (oracle/: fetd_oracle's adaptive BDF2 loop on a supernodal Cholesky with the same "
            "ordering, OpenMP + OpenBLAS on %d threads) on the %s %d-edge model: %s; not MKL PARDISO, which "
            "cannot be built here" % (threads, "reduced-resolution" if reduced else "full-resolution", om.n, how))
    return float(np.mean(vals)), info, text


def config3_media(m, seed: int = 3):
    """Config 3 on the config-1 mesh: the tet -> cell map of the 32 x 32 x 16
    inversion grid, the log-normal model (median 0.01 S/m, 0.5 decades) and
    the seeded perturbation (x 10^(0.1 N(0,1)) per cell) that makes the
    observations; conductivity per tet for both, permeability per tet."""
    from temf3dt_b200 import inversion, meshio
    grid = inversion.InversionGrid(INV_SHAPE, INV_BOX)
    cell = grid.tet_cells(m.mesh.nod_cor, m.mesh.tet_vex)
    sig0, mu = meshio.media_per_tet(m.mesh.tet_phy, m.ctl)
    earth = sig0 > 1e-6
    cell = np.where(earth, cell, -1)            # the grid lies below the surface; air tets keep 1e-12
    sc = inversion.lognormal_cells(grid.ncell, 0.01, 0.5, seed)
    sc_true = sc * 10.0 ** (0.1 * np.random.default_rng(seed + 30).standard_normal(grid.ncell))
    return dict(cell=cell, ncell=grid.ncell, mu=mu, sig=inversion.sigma_with_cells(sig0, cell, sc),
                sig_true=inversion.sigma_with_cells(sig0, cell, sc_true), cell_sigma=sc)


def adjoint_measure(local: int, fd_cells: int = 0):
    """Config 3: gradient of J = 1/2 sum (dBz/dt - d_obs)^2 over 64 receivers x
    40 gates with respect to log sigma of the 32 x 32 x 16 cells: a recorded
    forward run (eager launches, checkpoints every 50 solves) and the reverse
    sweep, both timed with CUDA events inside the library, against one
    forward run of the same model.  fd_cells > 0: central differences
    (log sigma +- 1e-3, the run's accept/reject decisions replayed) on that
    many seeded random cells."""
    from temf3dt_b200 import fetd, inversion
    m = model_for(3)
    c = m.ctl
    md = config3_media(m)
    args = (c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)
    with fetd.FetdGPU(local) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        g.set_media(md["sig_true"], md["mu"])
        g.assemble()
        o_true = g.run(*args)
        d_obs = inversion.gate_matrix(o_true.times, GATES) @ o_true.fields[:, :, 5]
        g.set_media(md["sig"], md["mu"])
        g.assemble()
        o_fwd = g.run(*args)
        g.adjoint_record(50)
        o = g.run(*args)
        J, dJ = inversion.dbdt_misfit(o.fields, o.times, GATES, d_obs)
        grad, _, tm = g.adjoint(dJ, md["cell"], md["ncell"])
        g.adjoint_record(0)
        out = {"ms": tm["ms_total"], "recorded_forward_ms": o.ms_total, "forward_ms": o_fwd.ms_total,
               "ratio_to_forward": tm["ms_total"] / o_fwd.ms_total, "factor_ms": tm["ms_factor"],
               "nodes": tm["nodes"], "blocks": tm["blocks"], "factorisations": tm["factors"],
               "launches": tm["launches"], "checkpoint_every": 50, "cells": md["ncell"],
               "cells_in_mesh": int(len(np.unique(md["cell"][md["cell"] >= 0]))), "misfit": J,
               "receivers": int(o.fields.shape[1]), "gates": len(GATES), "grad_finite": bool(np.isfinite(grad).all()),
               "model": "log-normal cells (median 0.01 S/m, 0.5 decades), observations of a 0.1-decade perturbation"}
        if fd_cells > 0:
            forced = o.trial_accepted.astype(np.int32)
            hit = np.unique(md["cell"][md["cell"] >= 0])
            pick = np.random.default_rng(32).choice(hit, size=min(fd_cells, len(hit)), replace=False)
            h = 1e-3
            scale = float(np.abs(grad).max())
            rel, fds, tol_used = [], [], []
            for k in pick:
                Jpm = []
                for sgn in (1.0, -1.0):
                    sig = md["sig"].copy()
                    sig[md["cell"] == k] *= np.exp(sgn * h)
                    g.set_media(sig, md["mu"])
                    g.assemble()
                    ok = g.run(*args, forced=forced)
                    Jpm.append(inversion.dbdt_misfit(ok.fields, ok.times, GATES, d_obs)[0])
                fd = (Jpm[0] - Jpm[1]) / (2 * h)
                fds.append(float(fd))
                rel.append(abs(fd - grad[k]) / max(abs(fd), 1e-300))
                # the GPU test's bound: 1e-4 relative, plus 1e-6 of the largest cell gradient
                tol_used.append(abs(fd - grad[k]) / (1e-4 * abs(fd) + 1e-6 * scale))
                print("fd cell %d: fd %.9e adjoint %.9e rel %.2e" % (k, fd, grad[k], rel[-1]),
                      file=sys.stderr, flush=True)
            out["fd"] = {"cells": [int(k) for k in pick], "max_rel_err": float(max(rel)),
                         "median_rel_err": float(np.median(rel)), "step": h, "grad_max": scale,
                         "fd": fds, "adjoint": [float(grad[k]) for k in pick],
                         "max_err_over_test_bound": float(max(tol_used))}
    return out


def config4_measure(local: int, max_steps: int):
    """Config 4: the ~5M-edge ellipsoid model with 256 small-loop sources in
    blocks of 64 columns.  Reports the analysis (nnz(L), factor flops), the
    device memory of the plan (one factor slot, relative indices, vectors)
    against the GPU's, and runs the first `max_steps` time steps of the
    adaptive loop for all 256 columns (each block of 64 one block sweep per
    step), timed with CUDA events inside the library."""
    import torch
    from temf3dt_b200 import fetd
    m = model_for(4)
    c = m.ctl
    free0, total = torch.cuda.mem_get_info(local)
    out = {"workload": CONFIGS[4]["label"], "tets": int(len(m.mesh.tet_vex)), "rhs": len(m.loops)}
    with fetd.FetdGPU(local) as g:
        t0 = time.perf_counter()
        info = fetd.load_case(g, m.mesh, m.ctl)
        out["setup_s"] = time.perf_counter() - t0
        st = g.stats()
        cols = m.source_columns(info["edg_vex"])
        rec_tet = g.locate(m.receivers, c.rec_charac)
        runs = []
        free1 = free0
        for b0 in range(0, len(cols), 64):   # the sources in blocks of 64 columns, one run each
            sel = [i for i in range(len(m.receivers)) if b0 <= m.rec_rhs[i] < b0 + 64]
            g.set_sources(cols[b0:b0 + 64], 1, c.pulse_type, c.t0, 1.0)
            g.set_receivers(rec_tet[sel], m.receivers[sel], rec_rhs=m.rec_rhs[sel] - b0)
            runs.append(g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum, max_steps=max_steps))
            free1 = min(free1, torch.cuda.mem_get_info(local)[0])
    ms = sum(o.ms_total for o in runs)
    steps_rhs = sum((len(o.steps) - 1) * 64 for o in runs)
    o = runs[0]
    out.update({"n_edges": int(st["n"]), "nnz_L": st["nnz_L"], "stored_doubles": st["stored"],
                "factor_slot_GB": 8 * st["stored"] / 1e9, "factor_tflop": st["flops"] / 1e12,
                "device_GB_in_use": (free0 - free1) / 1e9, "device_GB_total": total / 1e9,
                "steps_per_block": len(o.steps) - 1, "blocks": len(runs), "factorisations_per_block": o.n_factor,
                "ms_factor_each": o.ms_factor / max(o.n_factor, 1),
                "ms_per_step_64rhs": o.ms_steps / max(o.n_solve, 1),
                "steps_rhs_per_s": steps_rhs / (ms / 1e3), "ms_total": ms})
    return out


def batched_measure(local: int, plain_value: float, check_cols=(0, 27, 36, 63)):
    """Config 2: the 64 small loops on the config-1 mesh as one 64-column
    block per step, the full adaptive run (every factorisation included),
    after one warm-up run over the first 150 steps (autotuning, graph
    captures).  Against the plain single-RHS path on the same mesh (the
    headline value).  Accuracy: the columns in check_cols run again as plain
    single-RHS runs replaying the block run's accept/reject decisions; the
    largest dB/dt difference relative to each trace's maximum is reported."""
    from temf3dt_b200 import fetd
    m = model_for(2)
    c = m.ctl
    args = (c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)
    out = {}
    with fetd.FetdGPU(local) as g:
        info = fetd.load_case(g, m.mesh, m.ctl)
        st = g.stats()
        out["n_edges"] = int(st["n"])
        cols = m.source_columns(info["edg_vex"])
        rec_tet = g.locate(m.receivers, c.rec_charac)
        g.set_sources(cols, 1, c.pulse_type, c.t0, 1.0)
        g.set_receivers(rec_tet, m.receivers, rec_rhs=m.rec_rhs)
        g.run(*args, max_steps=150)
        ob = g.run(*args)
        batched = (len(ob.steps) - 1) * len(cols) / (ob.ms_total / 1e3)
        forced = ob.trial_accepted.astype(np.int32)
        errs = {}
        for k in check_cols:
            g.set_sources([cols[k]], 1, c.pulse_type, c.t0, 1.0)
            r = [i for i in range(len(m.receivers)) if m.rec_rhs[i] == k]
            g.set_receivers(rec_tet[r], m.receivers[r], rec_rhs=np.zeros(len(r), dtype=np.int32))
            o = g.run(*args, forced=forced)
            if not np.array_equal(o.steps, ob.steps):
                errs[int(k)] = float("inf")
                continue
            a, b = ob.fields[:, r, 3:6], o.fields[:, :, 3:6]
            errs[int(k)] = float(np.abs(a - b).max() / np.abs(b).max())
    ms_step = ob.ms_steps / max(ob.n_solve, 1)
    flops = (4 * st["nnz_L"] + 2 * st["nnz_A"]) * len(cols)
    return {**out, "value": batched, "unit": "steps*RHS/s", "rhs": len(cols), "plain_value": plain_value,
            "batched_over_plain": batched / plain_value, "steps": len(ob.steps) - 1,
            "factorisations": ob.n_factor, "ms_run": ob.ms_total, "ms_per_step_batched": ms_step,
            "ms_factor_batched": ob.ms_factor,
            "dbdt_rel_err_vs_plain": {"columns": errs, "max": max(errs.values()),
                                      "definition": "max |batched - plain| / max |plain| over the run, dB/dt"},
            "roofline": {"bound": "tensor", "unit": "TFLOP/s", "algorithmic_flops_per_step": flops,
                         "achieved": flops / (ms_step / 1e3) / 1e12,
                         "kernel": "one 64-column block step: BDF2 SpMM + persistent DMMA block sweeps + receivers"},
            "workload": CONFIGS[2]["label"] + ", full run"}


def layered_models(n_models: int = 16, seed: int = 5):
    """Independent 1-D layered models (3-6 layers, conductivities log-uniform
    in [1e-4, 1e-1] S/m, thicknesses log-uniform in [10, 300] m) on graded
    meshes of uneven size (mesh density drawn log-uniformly in [0.26, 1.5];
    with seed 5 the 16 meshes hold 101 525 to 986 423 edges)."""
    return [layered_model(i, sc) for i, sc in enumerate(layered_model_scales(n_models, seed))]


def layered_model_scales(n_models: int = 16, seed: int = 5):
    """The mesh-density scale of each layered model (log-uniform in [0.26, 1.5])."""
    rng = np.random.default_rng(seed)
    return [float(np.exp(rng.uniform(np.log(0.26), np.log(1.5)))) for _ in range(n_models)]


def layered_model(i: int, scale: float):
    """Layered model i of the batch (its own seed) at the given mesh scale."""
    from temf3dt_b200 import synth
    return synth.build_model("layered", seed=100 + i, scale=scale, ratio=2.0, **COMMON)


def models_measure(local: int, n_models: int = 16):
    """The layered models one after another (plain runs) against all of them
    in one lockstep batch with merged solve kernels (autotuned schedule).
    Unit: model time steps per second of the whole job."""
    from temf3dt_b200 import fetd
    models = layered_models(n_models)
    gs = []
    try:
        for m in models:
            g = fetd.FetdGPU(local)
            gs.append(g)
            fetd.load_case(g, m.mesh, m.ctl)
        c = models[0].ctl
        args = (c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)
        seq_ms, seq_steps = 0.0, 0
        for g in gs:
            g.run(*args)
            o = g.run(*args)
            seq_ms += o.ms_total
            seq_steps += len(o.steps) - 1
        with fetd.FetdBatch(gs) as b:
            b.run(*args, autotune=True)
            outs = b.run(*args)
            tm = b.timing()
            tu = b.tuning()
        bat_steps = sum(len(o.steps) - 1 for o in outs)
        sizes = [int(g.stats()["n"]) for g in gs]
    finally:
        for g in gs:
            g.close()
    seq = seq_steps / (seq_ms / 1e3)
    bat = bat_steps / (tm["ms_total"] / 1e3)
    return {"value": bat, "unit": "model-steps/s", "sequential_value": seq, "batch_over_sequential": bat / seq,
            "n_models": n_models, "edges_min": min(sizes), "edges_max": max(sizes), "edges_total": sum(sizes),
            "ms_batch": tm["ms_total"], "ms_sequential": seq_ms, "batch_factor_ms": tm["ms_factor"],
            "merged_solves": tm["merged_solves"], "tuning": tu}


def peak_value(peaks: dict, key: str, default: float) -> float:
    """A figure of MEASURED_PEAKS.json: a number, or an object holding one
    under "value" / "median" / "gbs"; the fallback when absent."""
    v = peaks.get(key)
    if isinstance(v, dict):
        v = next((v[k] for k in ("value", "median", "gbs") if k in v), None)
    try:
        return float(v) if v is not None and float(v) > 0 else default
    except (TypeError, ValueError):
        return default


def cpu_baseline(cfg: int, sample_steps: int) -> dict:
    """The GPU line's cpu_baseline: the reference arm's measurement as one
    scaled sample, run in a fresh process (no CUDA context, no torch threads)."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--config", str(cfg), "--steps", "1",
           "--warmup", "0", "--sample-steps", str(sample_steps)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800, env=env)
    except subprocess.TimeoutExpired:
        return {"value": None, "error": "CPU arm did not finish in 1800 s"}
    ref = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode == 0 and ref and "cpu_baseline" in ref[-1]:
        return ref[-1]["cpu_baseline"]
    why = ref[-1].get("unavailable") if ref else "exit %d: %s" % (r.returncode, r.stderr[-300:])
    return {"value": None, "error": "CPU arm: %s" % why}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = args.config
    try:
        value, info, text = cpu_arm(cfg, args.steps, args.warmup, args.sample_steps)
    except Exception as e:  # noqa: BLE001 - the arm reports why it could not run
        print(json.dumps({"impl": "reference", "unavailable": "CPU restatement failed: %s" % repr(e)[:300]}))
        return 0
    line = {
        "impl": "reference", "metric": "FETD steps*RHS/s", "value": value, "unit": "steps*RHS/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * info["seconds"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": CONFIGS[cfg]["label"], "n_edges": info["n_edges"],
                   "sample": "first %d time steps from rest per step, factorisation amortised" % info["steps"],
                   "reduced_model": info["reduced"]},
        "cpu_baseline": {"value": value, "unit": "steps*RHS/s", "cores": info["threads"], "kind": "port",
                         "sample": text},
        "e2e": {"value": value, "unit": "steps*RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from temf3dt_b200 import fetd
    cfg = args.config
    m = model_for(cfg)
    g = fetd.FetdGPU(local)
    t_setup = time.perf_counter()
    info = fetd.load_case(g, m.mesh, m.ctl)
    ncols = 1
    if cfg == 2:
        # batched: every loop is an RHS column; ranks take disjoint column blocks
        from temf3dt_b200.parallel import shard_range
        ev = info["edg_vex"]
        cols = m.source_columns(ev)
        lo, hi = shard_range(len(cols), world, rank)
        g.set_sources(cols[lo:hi], 1, m.ctl.pulse_type, m.ctl.t0, 1.0)
        sel = [i for i in range(len(m.receivers)) if lo <= m.rec_rhs[i] < hi]
        rt = g.locate(m.receivers[sel], m.ctl.rec_charac)
        g.set_receivers(rt, m.receivers[sel], rec_rhs=m.rec_rhs[sel] - lo)
        ncols = hi - lo
    t_setup = time.perf_counter() - t_setup
    st = g.stats()
    c = m.ctl
    plain = None
    if cfg == 2:
        # the plain single-RHS path on the same mesh (first loop, its receiver)
        g2 = fetd.FetdGPU(local)
        fetd.load_case(g2, m.mesh, m.ctl)
        g2.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)
        o2 = g2.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)
        plain = {"value": (len(o2.steps) - 1) / (o2.ms_total / 1e3), "unit": "steps*RHS/s", "rhs": 1,
                 "ms_per_run": o2.ms_total, "solve_ms_per_step": o2.ms_steps / max(o2.n_solve, 1)}
        g2.close()

    def one_run():
        return g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum)

    for _ in range(args.warmup):
        one_run()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    outs = []
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            outs.append(one_run())
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    dev_s = sum(o.ms_total for o in outs) / 1e3
    steps_run = sum(len(o.steps) - 1 for o in outs)
    t = torch.tensor([dev_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dev_s = float(t.item())
    value = steps_run * ncols * world / dev_s
    # --- e2e through the public API with host buffers ---
    from temf3dt_b200 import meshio
    sig, mu = meshio.media_per_tet(m.mesh.tet_phy, c)
    e2e_times = []
    h2d = sig.nbytes + mu.nbytes
    d2h = 0
    for k in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.set_media(sig, mu)
        g.assemble()
        o = one_run()
        d2h = o.fields.nbytes + o.steps.nbytes + o.times.nbytes + o.dts.nbytes
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e_steps = len(o.steps) - 1
    e2e_val = e2e_steps * ncols * world / float(np.mean(e2e_times))
    # --- the other configs of the metric, beside the headline (one GPU) ---
    #   batched: config 2 (64 loops on this mesh as one block, full run) against this line's value
    #   models:  16 layered models of uneven size, one after another and as one batch
    #   adjoint: config 3 (log-normal cells on this mesh), one gradient against one forward run
    adj = models = batched = None
    if cfg == 1 and world == 1:
        g.close()
        g = None
        if args.batched:
            batched = batched_measure(local, value)
        if args.models > 0:
            models = models_measure(local, args.models)
        if args.adjoint:
            adj = adjoint_measure(local)
    # --- roofline of the dominant phase ---
    o = outs[-1]
    ms_fac = o.ms_factor / max(o.n_factor, 1)
    ms_step = o.ms_steps / max(o.n_solve, 1)
    fac_share = o.ms_factor / o.ms_total
    dgemm = measured_dgemm_tflops(torch)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peak_value(peaks, "hbm_gbs", 6650.0)
    factor_rate = st["flops"] / (ms_fac / 1e3) / 1e12
    if cfg == 2:
        # the 64-column block step is a DMMA contraction: 4 nnz(L) flops per
        # column for both sweeps plus 2 nnz(A) for the SpMV
        flops = (4 * st["nnz_L"] + 2 * st["nnz_A"]) * ncols
        ach = flops / (ms_step / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": dgemm, "unit": "TFLOP/s", "frac": ach / dgemm,
                "traffic": None, "algorithmic_flops_per_step": flops,
                "kernel": "one 64-column block step: BDF2 SpMM + persistent DMMA block sweeps + receivers",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)",
                "factor": {"achieved_tflops": factor_rate, "peak_dgemm_tflops": dgemm, "frac": factor_rate / dgemm}}
    elif fac_share >= 0.5:
        roof = {"bound": "tensor", "achieved": factor_rate, "peak": dgemm, "unit": "TFLOP/s",
                "frac": factor_rate / dgemm, "traffic": None,
                "kernel": "numeric supernodal LL^T (potrf/trsm + DMMA update levels)",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)"}
    else:
        # algorithmic bytes of one time step: both sweeps read the whole factor,
        # plus the BDF2 SpMV (values + column indices, row pointers, 3 vectors)
        nbytes = 2 * 8 * st["nnz_L"] + 12 * st["nnz_A"] + 4 * st["n"] + 24 * st["n"]
        ach = nbytes / (ms_step / 1e3) / 1e9
        # DRAM bytes per step scaled from the ncu capture of the same sweep
        # kernels on the config-0 model (dram__bytes_read + write per launch):
        # 1.047 (forward) and 1.077 (backward) x the stored panel bytes
        traffic = (1.047 + 1.077) * 8 * st["stored"] + 12 * st["nnz_A"] + 28 * st["n"]
        roof = {"bound": "hbm", "achieved": ach / 1.0, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": traffic,
                "kernel": "one time step: BDF2 SpMV + persistent forward/backward supernodal sweeps + receivers",
                "algorithmic_bytes_per_step": nbytes,
                "peak_source": ("MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm != 6650.0
                                else "fallback 6.65 TB/s (of fallback)"),
                "factor": {"achieved_tflops": factor_rate, "peak_dgemm_tflops": dgemm, "frac": factor_rate / dgemm}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(cfg, args.sample_steps or 10)
    line = {
        "metric": "FETD steps*RHS/s", "value": value, "unit": "steps*RHS/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded graded hex mesh)",
        "config": {"workload": CONFIGS[cfg]["label"], "n_edges": int(st["n"]), "nnz_L": st["nnz_L"],
                   "factor_tflop": st["flops"] / 1e12, "rhs_per_rank": ncols, "time_steps_per_run": len(o.steps) - 1,
                   "factorisations_per_run": o.n_factor, "parallelism": "replicas" if cfg != 2 else "rhs-columns",
                   "l2": "inputs larger than L2 (factors of GBs), no flush"},
        "e2e": {"value": e2e_val, "unit": "steps*RHS/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(sum(x.n_launch for x in outs)),
        "plain_same_mesh": plain,
        "batched_over_plain": (value / world / plain["value"]) if plain else None,
        "adjoint": adj,
        "batched": batched,
        "models": models,
        "phases_ms_per_run": {"factor": o.ms_factor, "steps": o.ms_steps, "total": o.ms_total,
                              "factor_each": ms_fac, "solve_step_each": ms_step, "setup_s": t_setup},
    }
    if rank == 0:
        print(json.dumps(line))
    if g is not None:
        g.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def profile_run(args):
    """--profile-steps N: the first N time steps of the config's model (its
    factorisations included), for profiler captures; prints the phase
    timings.  Not a bench line (no warm-up, part of a run).  With --timeline,
    one single-column solve with per-task GPU timestamps instead, summarised
    per phase of the tree (for the sweep kernels)."""
    from temf3dt_b200 import fetd, synth
    if args.h_core > 0:
        kw = dict(CONFIGS[args.config]["kw"], **COMMON)
        kw["h_core"] = args.h_core
        m = synth.build_model(CONFIGS[args.config]["kind"], seed=args.config, **kw)
    else:
        m = model_for(args.config)
    c = m.ctl
    with fetd.FetdGPU(0) as g:
        info = fetd.load_case(g, m.mesh, m.ctl)
        if args.replicate > 1:
            # the single loop as this many identical RHS columns
            cols = [(info["src_edg"], info["src_drc"])] * args.replicate
            g.set_sources(cols, c.source_type, c.pulse_type, c.t0, c.current)
            g.set_receivers(np.repeat(info["rec_tet"], args.replicate), np.repeat(c.rec_cor, args.replicate, axis=0),
                            rec_rhs=np.arange(args.replicate))
        elif args.config == 2:
            cols = m.source_columns(info["edg_vex"])
            k = len(cols) if args.rhs <= 0 else min(args.rhs, len(cols))
            g.set_sources(cols[:k], 1, c.pulse_type, c.t0, 1.0)
            sel = [i for i in range(len(m.receivers)) if m.rec_rhs[i] < k]
            g.set_receivers(g.locate(m.receivers[sel], c.rec_charac), m.receivers[sel], rec_rhs=m.rec_rhs[sel])
        st = g.stats()
        if args.solve_only > 0:
            # one factorisation and K single-column solves with the analysis's
            # default plan (no tuning): the sweep kernels launch 4 K times only
            g.factor(1, c.t0 / c.sp_division)
            b = np.random.default_rng(0).standard_normal(int(st["n"]))
            for _ in range(args.solve_only):
                x = g.solve(1, b)
            print(json.dumps({"config": args.config, "plan": g.solve_plan(), "stored": st["stored"],
                              "finite": bool(np.isfinite(x).all())}))
            return 0
        if args.timeline:
            g.factor(1, c.t0 / c.sp_division)
            split, cand = g.tune_solve(1, 1)
            if args.plans:
                # forced plans "level,split,options;...": sweep spans of each (median of 3)
                tuned = g.solve_plan()
                spans = {}
                for spec in args.plans.split(";"):
                    lv, sp, op = (int(v) for v in spec.split(","))  # op: run leaders 0/1
                    g.set_solve_plan(lv, min(sp, int(st["levels"])), bool(op & 1))
                    rs = []
                    for _ in range(3):
                        f, b = g.solve_timeline(1)
                        rs.append(((f[:, 2].max() - f[:, 0].min()) / 1e3, (b[:, 2].max() - b[:, 0].min()) / 1e3))
                    rs.sort(key=lambda v: v[0] + v[1])
                    spans[spec] = {"fwd_us": rs[1][0], "bwd_us": rs[1][1]}
                print(json.dumps({"config": args.config, "tuned": tuned, "cand": cand, "plans": spans}))
                g.set_solve_plan(tuned["tree_level"], tuned["split"], tuned["run_leaders"])
            f, b = g.solve_timeline(1)
            if args.timeline_out:
                np.savez_compressed(args.timeline_out, forward=f, backward=b)
            out = {"config": args.config, "stats": st, "plan": g.solve_plan(), "split_candidates_ms": cand}
            names = {0: "diagonal", 1: "chunk", 2: "subtree", 3: "leader"}
            for name, T in (("forward", f), ("backward", b)):
                t0 = T[:, 0].min()
                span = (T[:, 2].max() - t0) / 1e3
                kinds = {}
                for k in np.unique(T[:, 5]):
                    R = T[T[:, 5] == k]
                    kinds[names.get(int(k), str(k))] = {
                        "tasks": int(len(R)), "first_start_us": float((R[:, 0].min() - t0) / 1e3),
                        "last_end_us": float((R[:, 2].max() - t0) / 1e3),
                        "work_us_mean": float(np.mean(R[:, 2] - R[:, 1]) / 1e3),
                        "to_ready_us_mean": float(np.mean(R[:, 1] - R[:, 0]) / 1e3)}
                # time by which each level's tasks (not the subtrees) have all ended
                tk = T[T[:, 5] != 2]
                lev = tk[:, 7]
                levels = np.unique(lev)
                ends = np.array([tk[lev == l, 2].max() - t0 for l in levels]) / 1e3
                done = np.maximum.accumulate(ends if name == "forward" else ends[::-1]) if len(ends) else ends
                q = {p_: float(done[int(p_ / 100 * (len(done) - 1))]) for p_ in (10, 25, 50, 75, 100)} if len(done) else {}
                out[name] = {"tasks": int(len(T)), "span_us": float(span), "task_levels": int(len(levels)),
                             "levels_done_us_at_pct": q, "by_kind": kinds}
            print(json.dumps(out))
            return 0
        o = g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum, max_steps=args.profile_steps)
        print(json.dumps({"config": args.config, "stats": st, "rows": len(o.steps), "ms_factor": o.ms_factor,
                          "n_factor": o.n_factor, "ms_steps": o.ms_steps, "n_solve": o.n_solve,
                          "ms_per_solve": o.ms_steps / max(o.n_solve, 1), "ms_total": o.ms_total}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 3, 4],
                    help="3: the adjoint measurement of config 3 alone; 4: the 5M-edge 256-source run "
                         "(one JSON object each, not a bench line)")
    ap.add_argument("--c4-steps", type=int, default=100, help="config 4: time steps to run")
    ap.add_argument("--sample-steps", type=int, default=0, help="CPU arm: time steps per sample (0: 10)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--adjoint", type=int, default=1, help="config 1: also time one config-3 adjoint gradient")
    ap.add_argument("--models", type=int, default=16,
                    help="config 1: also run this many layered models one by one and as one batch")
    ap.add_argument("--batched", type=int, default=1,
                    help="config 1: also run config 2 (64 loops as one 64-column block) on the same mesh")
    ap.add_argument("--fd-cells", type=int, default=0,
                    help="config 3: central differences on this many random cells beside the gradient")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="profiling: run only the first N time steps of the config's model and print phase timings")
    ap.add_argument("--timeline", action="store_true", help="profiling: one solve with per-task GPU timestamps")
    ap.add_argument("--timeline-out", default="", help="profiling: also save the raw timeline rows (.npz)")
    ap.add_argument("--plans", default="", help="profiling, with --timeline: sweep spans of forced plans "
                    "'level,split,leaders;...' (leaders 0/1)")
    ap.add_argument("--solve-only", type=int, default=0,
                    help="profiling: one factorisation and this many single-column solves (default plan)")
    ap.add_argument("--rhs", type=int, default=0, help="profiling, config 2: the first RHS loops only (0 = all)")
    ap.add_argument("--h-core", type=float, default=0.0, help="profiling: core cell size override (m)")
    ap.add_argument("--replicate", type=int, default=1,
                    help="profiling: solve the config's loop as this many identical RHS columns")
    args = ap.parse_args()
    if args.profile_steps > 0 or args.timeline or args.solve_only > 0:
        return profile_run(args)
    if args.impl == "reference":
        return reference_arm(args)
    if args.config == 4:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"config4": config4_measure(int(os.environ.get("LOCAL_RANK", "0")), args.c4_steps)}))
        return 0
    if args.config == 3:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"config": CONFIGS[3]["label"],
                          "adjoint": adjoint_measure(int(os.environ.get("LOCAL_RANK", "0")), args.fd_cells)}))
        return 0
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
