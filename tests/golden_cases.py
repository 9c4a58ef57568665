"""Helpers shared by the tests: load golden fixtures, build oracle models and
GPU models for the same inputs."""
from __future__ import annotations

import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import fetd_oracle as O  # noqa: E402
from temf3dt_b200 import meshio  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")


def load_fixture(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def _cntl_file(text: str) -> str:
    fd, path = tempfile.mkstemp(suffix=".cntl")
    with os.fdopen(fd, "w") as fh:
        fh.write(str(text))
    return path


def oracle_control(fx: dict) -> O.Control:
    path = _cntl_file(fx["cntl"])
    try:
        return O.read_cntl(path)
    finally:
        os.unlink(path)


def host_control(fx: dict) -> meshio.Control:
    path = _cntl_file(fx["cntl"])
    try:
        return meshio.read_cntl(path)
    finally:
        os.unlink(path)


def fixture_mesh_dict(fx: dict) -> dict:
    return dict(nod_cor=fx["nod_cor"], tet_vex=fx["tet_vex"].astype(np.int64), tet_phy=fx["tet_phy"].astype(np.int64),
                src_vex=fx["src_vex"].astype(np.int64), src_phy=fx["src_phy"].astype(np.int64))


def fixture_mesh(fx: dict) -> meshio.Mesh:
    d = fixture_mesh_dict(fx)
    return meshio.Mesh(d["nod_cor"], d["tet_vex"], d["tet_phy"], d["src_vex"], d["src_phy"])


def sigma_rescale_factor(sig_dom) -> float:
    """src_small's sig_parameter (src_small/FETD_FWD.f90:314-323): 1 / sigma of
    the last domain read (the earth in the shipped example)."""
    return 1.0 / float(sig_dom[-1])


def output_scale(p: float) -> float:
    """src_small/FETD_FWD.f90:1526: a_f / p**2 * pi**log10(p)."""
    return float(np.pi ** np.log10(p) / p ** 2)


def oracle_model_from_fixture(fx: dict, sigma_rescale: bool = False):
    ctl = oracle_control(fx)
    scale = 1.0
    if sigma_rescale:
        p = sigma_rescale_factor(ctl.sig_dom)
        ctl.sig_dom = ctl.sig_dom.copy()
        ctl.sig_dom[1:] = ctl.sig_dom[1:] * p
        scale = output_scale(p)
    return O.build_model(fixture_mesh_dict(fx), ctl), scale


def host_model_from_fixture(fx: dict, sigma_rescale: bool = False):
    ctl = host_control(fx)
    scale = 1.0
    if sigma_rescale:
        p = sigma_rescale_factor([d[1] for d in ctl.domains])
        ctl.domains = [ctl.domains[0]] + [(d[0], d[1] * p, d[2], d[3]) for d in ctl.domains[1:]]
        scale = output_scale(p)
    return fixture_mesh(fx), ctl, scale


def synth_oracle_model(model) -> O.OracleModel:
    """Oracle model for a temf3dt_b200.synth.Model (same arrays)."""
    c = model.ctl
    oc = O.Control(rec_cor=c.rec_cor, rec_charac=c.rec_charac,
                   dom_ind=np.array([d[0] for d in c.domains]), sig_dom=np.array([d[1] for d in c.domains]),
                   per_dom=np.array([d[2] for d in c.domains]) * O.EPS0,
                   mag_dom=np.array([d[3] for d in c.domains]) * O.MU0,
                   src_num=1, src_sourcetype=c.source_type, src_pulsetype=c.pulse_type, src_pulsewidth=c.t0,
                   src_current=c.current, step_mthd=2, step_dvsi=c.sp_division, time_maxm=c.time_maximum,
                   step_dble=c.sp_double, step_dblesize=c.sp_dblesize, o_f=c.output, time_channels=c.time_points)
    mesh = dict(nod_cor=model.mesh.nod_cor, tet_vex=model.mesh.tet_vex, tet_phy=model.mesh.tet_phy,
                src_vex=model.mesh.src_vex, src_phy=model.mesh.src_phy)
    return O.build_model(mesh, oc)


def small_synth(**kw):
    """A small synthetic half-space model (~37k edges) used by the parity tests."""
    from temf3dt_b200 import synth
    args = dict(h_core=250, ratio=2.5, h_z=50, z_core=150, sp_double=20, time_maximum=2e-4)
    args.update(kw)
    return synth.build_model("halfspace", **args)


def tiny_synth(**kw):
    """A tiny synthetic model (~5k edges) for quick oracle runs."""
    from temf3dt_b200 import synth
    args = dict(radius=200.0, h_core=200, ratio=3.0, h_z=100, z_core=100, half=20000.0, sp_double=8,
                sp_division=4, time_maximum=2e-5)
    args.update(kw)
    return synth.build_model("halfspace", **args)


def cell_grid_2x2x2(om) -> "np.ndarray":
    """Inversion cells for the adjoint tests: a 2 x 2 x 2 grid of 400 x 400 x
    150 m cells under the loop; 0-based cell per tet, -1 outside."""
    X = om.nod_cor[om.tet_vex - 1].mean(axis=1)
    cell = -np.ones(len(X), dtype=np.int64)
    ins = (np.abs(X[:, 0]) < 400) & (np.abs(X[:, 1]) < 400) & (X[:, 2] > 0) & (X[:, 2] < 300)
    ix = ((X[:, 0] + 400) // 400).astype(int)
    iy = ((X[:, 1] + 400) // 400).astype(int)
    iz = (X[:, 2] // 150).astype(int)
    cell[ins] = (ix * 4 + iy * 2 + iz)[ins]
    return cell


def adjoint_misfit_case(rows, seed: int = 0):
    """Observed data = the run's own output with 5 % multiplicative noise, and
    weights 1/max|.|^2 on the dB/dt and b columns (9 output columns)."""
    rng = np.random.default_rng(seed)
    d_obs = rows * (1 + 0.05 * rng.standard_normal(rows.shape))
    mask = np.zeros_like(d_obs)
    mask[:, :, 3:9] = 1.0 / np.maximum(np.abs(rows[:, :, 3:9]).max(axis=0), 1e-300) ** 2
    return d_obs, mask


# anisotropic variant of the tiny model: the earth gets a rotated conductivity
# tensor and unequal (unrotated) relative permeabilities; air stays isotropic
ANISO_EARTH = ((1e-3, 2e-3, 5e-4), (10.0, 20.0, 30.0))
ANISO_EARTH_MU = ((1.0, 1.2, 0.9), (0.0, 0.0, 0.0))


def aniso_controls(model, bound_cond: int = 1):
    """(host Control, oracle Control) of a synthetic model with anisotropic
    media in the earth and the given boundary condition."""
    import copy
    import math
    from temf3dt_b200 import meshio as MI
    hc = copy.deepcopy(model.ctl)
    hc.aniso_domains = []
    for phys, sig, epsr, mur in hc.domains:
        if sig > 1e-6:
            hc.aniso_domains.append((phys, ANISO_EARTH, ((1.0,) * 3, (0.0,) * 3), ANISO_EARTH_MU))
        else:
            hc.aniso_domains.append((phys, ((sig,) * 3, (0.0,) * 3), ((epsr,) * 3, (0.0,) * 3), ((mur,) * 3, (0.0,) * 3)))
    hc.domains = []
    hc.bound_cond = bound_cond
    oc = copy.copy(synth_oracle_model_control(model))
    oc.aniso = True
    oc.bound_cond = bound_cond
    d2r = math.pi / 180.0
    oc.dom_ind = np.array([d[0] for d in hc.aniso_domains])
    oc.sig_ani = np.array([d[1][0] for d in hc.aniso_domains])
    oc.sig_ang = np.array([d[1][1] for d in hc.aniso_domains]) * d2r
    oc.per_ani = np.array([d[2][0] for d in hc.aniso_domains])
    oc.per_ang = np.array([d[2][1] for d in hc.aniso_domains]) * d2r
    oc.mag_ani = np.array([d[3][0] for d in hc.aniso_domains])
    oc.mag_ang = np.array([d[3][1] for d in hc.aniso_domains]) * d2r
    assert isinstance(MI.Control(), type(hc))
    return hc, oc


def synth_oracle_model_control(model) -> O.Control:
    """The oracle Control of a synthetic model (isotropic, as built)."""
    c = model.ctl
    return O.Control(rec_cor=c.rec_cor, rec_charac=c.rec_charac,
                     dom_ind=np.array([d[0] for d in c.domains]), sig_dom=np.array([d[1] for d in c.domains]),
                     per_dom=np.array([d[2] for d in c.domains]) * O.EPS0,
                     mag_dom=np.array([d[3] for d in c.domains]) * O.MU0,
                     src_num=1, src_sourcetype=c.source_type, src_pulsetype=c.pulse_type, src_pulsewidth=c.t0,
                     src_current=c.current, step_mthd=2, step_dvsi=c.sp_division, time_maxm=c.time_maximum,
                     step_dble=c.sp_double, step_dblesize=c.sp_dblesize, o_f=c.output, time_channels=c.time_points)


def oracle_model_with(model, oc):
    mesh = dict(nod_cor=model.mesh.nod_cor, tet_vex=model.mesh.tet_vex, tet_phy=model.mesh.tet_phy,
                src_vex=model.mesh.src_vex, src_phy=model.mesh.src_phy)
    return O.build_model(mesh, oc)


def golden_field_report(steps, times, dbz, trial_errors, gold, sp_double, rtol=6e-4):
    """Row-by-row comparison of a run with a shipped .field (step, time, dB_z/dt
    printed to 4 digits).  Returns (first row whose time differs, or the row
    count when none does; the trial error that decided that row, or None;
    largest relative dB_z/dt difference over the agreeing rows, away from the
    sign change).  Trial k runs at step (k+1) * sp_double
    (src/FETD_FWD.f90:1312), so the first row after a differing decision is
    decided by the last trial at or before it."""
    n = min(len(times), len(gold))
    same = np.isclose(np.asarray(times[:n]), gold[:n, 1], rtol=rtol, atol=0) | (gold[:n, 1] == 0)
    first = int(np.argmin(same)) if not same.all() else n
    if first == n and len(times) != len(gold):
        first = n            # one run ends earlier: the rows after n differ
    decided = None
    if first < max(len(times), len(gold)) and len(trial_errors):
        step = int(steps[min(first, len(steps) - 1)])
        k = step // sp_double - 1
        if 0 <= k < len(trial_errors):
            decided = float(trial_errors[k])
    gd = gold[:first, 2]
    v = np.asarray(dbz[:first])
    big = np.abs(gd) >= 1e-3 * np.abs(gd).max()
    rel = float((np.abs(v[big] - gd[big]) / np.abs(gd[big])).max()) if big.any() else 0.0
    return first, decided, rel


def golden_decisions(gold, sp_double):
    """The accept/reject decisions of the run that wrote a .field, read off its
    time column: trial k runs at step (k+1) * sp_double and was accepted iff the
    time step after it is about twice the one before it (src/FETD_FWD.f90:1404-1418)."""
    t = gold[:, 1]
    out = []
    s = sp_double
    while s + 1 < len(t):
        before = t[s - 1] - t[s - 2]
        after = t[s + 1] - t[s]
        out.append(bool(after > 1.5 * before))
        s += sp_double
    return out


def free_divergence_explained(k, gpu_error, oracle_errors, file_decisions):
    """Whether a free GPU run may part from a shipped .field at trial k.

    The file's build decided trial k by its own estimate; the oracle's
    estimates (the file's own decision history replayed) stand in for it.
    Either the restated rule itself disagrees with the file at k (the oracle's
    estimate, with the file's not_changed count, falls on the other side of
    1e-4: the reference build's own rounding decided it), or the GPU's and
    the oracle's estimates lie on both sides of 1e-4 or further apart than
    the oracle's is from it (solver rounding in the air fields that dominate
    the late estimates)."""
    ora = float(oracle_errors[k])
    not_changed = 0
    for d in file_decisions[:k]:
        not_changed = 0 if d else not_changed + 1
    oracle_accepts = not (ora > 1e-4 and not_changed < 2)  # src/FETD_FWD.f90:1382
    if oracle_accepts != file_decisions[k]:
        return True
    return (gpu_error - 1e-4) * (ora - 1e-4) < 0 or abs(gpu_error - ora) >= abs(ora - 1e-4)
