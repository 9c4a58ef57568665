"""Run the first N time steps of a benchmark model, for profiler captures.

    python -m temf3dt_b200.profile_case --config 0 --max-steps 150
    python -m temf3dt_b200.profile_case --config 2 --max-steps 150   # 64 loops = 64 RHS columns

Builds the same seeded synthetic model as ``bench.py --config K``, assembles
and analyses it, and runs the FETD time loop for the first ``max-steps``
steps (the factorisations and trials those steps contain included).  It prints
the phase timings; it is not a benchmark (no warm-up, not the whole run).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import fetd, synth

CONFIG_KW = {
    0: ("halfspace", dict(h_core=125, ratio=2.0, h_z=25)),
    1: ("block", dict()),
    2: ("multiloop", dict()),
}
COMMON = dict(t0=1e-6, sp_division=10, sp_double=100, time_maximum=1e-2)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=0, choices=sorted(CONFIG_KW))
    ap.add_argument("--max-steps", type=int, default=150)
    ap.add_argument("--rhs", type=int, default=0, help="multiloop: use the first RHS loops only (0 = all)")
    ap.add_argument("--scale", type=float, default=1.0, help="grid-line density factor (< 1: smaller mesh)")
    ap.add_argument("--h-core", type=float, default=0.0, help="core cell size override (m)")
    ap.add_argument("--replicate", type=int, default=1,
                    help="single-loop models: solve the loop as this many identical RHS columns")
    a = ap.parse_args()
    kind, kw = CONFIG_KW[a.config]
    kw = dict(kw)
    kw.update(COMMON)
    if a.h_core > 0:
        kw["h_core"] = a.h_core
    m = synth.build_model(kind, seed=a.config, scale=a.scale, **kw)
    with fetd.FetdGPU(0) as g:
        info = fetd.load_case(g, m.mesh, m.ctl)
        if kind == "multiloop":
            # every loop is a right-hand-side column with its own receiver
            cols = m.source_columns(info["edg_vex"])
            k = len(cols) if a.rhs <= 0 else min(a.rhs, len(cols))
            g.set_sources(cols[:k], 1, m.ctl.pulse_type, m.ctl.t0, 1.0)
            sel = [i for i in range(len(m.receivers)) if m.rec_rhs[i] < k]
            g.set_receivers(g.locate(m.receivers[sel], m.ctl.rec_charac), m.receivers[sel], rec_rhs=m.rec_rhs[sel])
        elif a.replicate > 1:
            cols = [(info["src_edg"], info["src_drc"])] * a.replicate
            g.set_sources(cols, m.ctl.source_type, m.ctl.pulse_type, m.ctl.t0, m.ctl.current)
            g.set_receivers(np.repeat(info["rec_tet"], a.replicate), np.repeat(m.ctl.rec_cor, a.replicate, axis=0),
                            rec_rhs=np.arange(a.replicate))
        st = g.stats()
        out = g.run(m.ctl.sp_division, m.ctl.sp_double, m.ctl.sp_dblesize, m.ctl.time_maximum,
                    max_steps=a.max_steps)
        print(json.dumps({"config": a.config, "stats": st, "rows": len(out.steps), "ms_factor": out.ms_factor,
                          "n_factor": out.n_factor, "ms_steps": out.ms_steps, "n_solve": out.n_solve,
                          "ms_per_solve": out.ms_steps / max(out.n_solve, 1), "ms_total": out.ms_total}))


if __name__ == "__main__":
    main()
