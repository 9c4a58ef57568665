"""Build the golden fixtures under tests/golden/ from the reference checkout.

Run here (where the reference is mounted) with
    python tests/golden/make_golden.py --reference PATH [--oracle] [--linux-oracle]
It packs, for each shipped example of the reference, the mesh (.mesh), the
control file (.cntl, as text) and the shipped output (.field rows) into one
compressed .npz, so the GPU tests can run the reference's own examples
without the reference checkout.  With --oracle it also runs the CPU oracle on
the src_small example (sigma rescaled as that build does) and stores its
rows and trial decisions.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    # fixture name: path of the example root within the reference
    "linux_mod_big": "LINUX/mod_big_sig_0.001",
    "linux_mod_small": "LINUX/mod_small_sig_0.001",
    "src_small_mod_small": "src_small/mod_small_sig_0.001",
}


def pack(ref: str, name: str, rel: str) -> str:
    from oracle import fetd_oracle as O
    root = os.path.join(ref, rel)
    mesh = O.read_mesh(root + ".mesh")
    with open(root + ".cntl") as fh:
        cntl = fh.read()
    field = O.read_field(root + ".field")
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, nod_cor=mesh["nod_cor"], tet_vex=mesh["tet_vex"].astype(np.int32),
                        tet_phy=mesh["tet_phy"].astype(np.int16), src_vex=mesh["src_vex"].astype(np.int32),
                        src_phy=mesh["src_phy"].astype(np.int16), cntl=np.array(cntl), field=field,
                        source=np.array(rel))
    return out


def oracle_src_small(max_rows: int = 700) -> str:
    """Oracle run on the src_small example with that build's sigma rescaling
    (src_small/FETD_FWD.f90:314-328): earth sigma / sigma_earth, output scaled by
    pi**log10(p) / p**2 with p = 1/sigma_earth (src_small/FETD_FWD.f90:1526)."""
    from tests.golden_cases import load_fixture, oracle_model_from_fixture
    fx = load_fixture("src_small_mod_small")
    om, scale = oracle_model_from_fixture(fx, sigma_rescale=True)
    from oracle import fetd_oracle as O
    res = O.run_fetd(om, max_steps=max_rows)
    out = os.path.join(HERE, "oracle_src_small.npz")
    np.savez_compressed(out, steps=np.array(res.steps), times=np.array(res.times), dts=np.array(res.dts),
                        fields=res.fields, trial_errors=np.array(res.trial_errors),
                        trial_accepted=np.array(res.trial_accepted), output_scale=scale)
    return out


def oracle_linux(name: str) -> str:
    """Oracle run of a LINUX example (from its fixture) with the schedule rule
    of the build that wrote the shipped .field (legacy_linux) and the file's
    own accept/reject decisions (read off its time column), on the CPU
    supernodal Cholesky: the decisions, the oracle's trial errors on that
    history, and its rows (step, time, dB_z/dt).  A GPU test replays the same
    decisions and compares every row with the file, and uses the trial errors
    to tell a decision that FP64 solver rounding can flip (late trials, whose
    error estimate is dominated by the poorly determined air fields) from a
    real difference."""
    from oracle import supernodal_cpu as SN
    from oracle import fetd_oracle as O
    from tests.golden_cases import golden_decisions, load_fixture, oracle_control, oracle_model_from_fixture
    SN.build()
    fx = load_fixture(name)
    om, _ = oracle_model_from_fixture(fx)
    forced = golden_decisions(fx["field"], oracle_control(fx).step_dble)
    res = O.run_fetd(om, legacy_linux=True, slots=SN.SupernodalSlots(om), forced=forced)
    out = os.path.join(HERE, "oracle_" + name + ".npz")
    np.savez_compressed(out, steps=np.array(res.steps), times=np.array(res.times),
                        dbz=np.asarray(res.fields)[:, 0, 5], trial_errors=np.array(res.trial_errors),
                        trial_accepted=np.array(res.trial_accepted))
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", help="root of the reference checkout (packs the fixtures)")
    ap.add_argument("--oracle", action="store_true", help="also the oracle run of the src_small example")
    ap.add_argument("--linux-oracle", action="store_true",
                    help="the oracle runs of the LINUX examples, from their fixtures (no reference needed)")
    a = ap.parse_args()
    if not a.reference and not a.linux_oracle:
        ap.error("--reference is required unless only --linux-oracle is given")
    if a.reference:
        for name, rel in CASES.items():
            print(pack(a.reference, name, rel))
        if a.oracle:
            print(oracle_src_small())
    if a.linux_oracle:
        for name in ("linux_mod_big", "linux_mod_small"):
            print(oracle_linux(name))
