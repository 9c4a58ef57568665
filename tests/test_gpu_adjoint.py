"""GPU adjoint gradient through the C ABI: against the oracle adjoint on the
same solve graph, against finite differences of GPU runs, and independent of
the checkpoint interval.  Marked ``gpu``; run on a B200.

Tolerances (FP64): the GPU and oracle states differ by about 1e-12 of their
scale (different factorisation orderings), so the gradients agree to 1e-8 of
the largest cell gradient; central differences with h = 1e-3 in log(sigma)
carry an O(h^2) truncation, checked at 1e-4.
"""
import numpy as np
import pytest

from oracle import fetd_adjoint as AD
from temf3dt_b200 import fetd
from tests.golden_cases import adjoint_misfit_case, cell_grid_2x2x2, small_synth, synth_oracle_model, tiny_synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tiny():
    m = tiny_synth(time_maximum=1e-5)
    om = synth_oracle_model(m)
    gr, states, rows = AD.forward_graph(om)
    g = fetd.FetdGPU(0)
    info = fetd.load_case(g, m.mesh, m.ctl)
    yield m, om, gr, states, rows, g, info
    g.close()


@pytest.fixture(scope="module")
def small():
    m = small_synth()
    om = synth_oracle_model(m)
    g = fetd.FetdGPU(0)
    info = fetd.load_case(g, m.mesh, m.ctl)
    yield m, om, g, info
    g.close()


def _run(m, g, **kw):
    return g.run(m.ctl.sp_division, m.ctl.sp_double, m.ctl.sp_dblesize, m.ctl.time_maximum, **kw)


def test_adjoint_matches_oracle(tiny):
    m, om, gr, states, rows, g, info = tiny
    g.adjoint_record(7)
    out = _run(m, g, forced=np.array(gr.decisions, dtype=np.int32))
    assert np.array_equal(out.trial_accepted, np.array(gr.decisions))
    assert np.abs(out.fields - rows).max() <= 1e-8 * np.abs(rows).max()
    d_obs, mask = adjoint_misfit_case(rows)
    dJ9 = mask * (out.fields - d_obs)
    cell = cell_grid_2x2x2(om)
    gc, gt, tm = g.adjoint(dJ9, cell, 8)
    dJ = AD.fields_grad_to_samples(dJ9, gr.row_step, gr.row_dt)
    ref, ref_t = AD.adjoint_gradient(om, gr, states, dJ, cell, 8, per_tet=True)
    assert tm["nodes"] == gr.n_nodes
    assert np.abs(gc - ref).max() <= 1e-8 * np.abs(ref).max(), (gc, ref)
    # per tet as dJ/dlog(sigma_t): dJ/dsigma_t of the 1e-12 S/m air tets is
    # large and set by cancellation in 3x_k - 4x_a + x_b, but weighs nothing
    sg = info["sig"]
    assert np.abs(sg * (gt - ref_t)).max() <= 1e-8 * np.abs(sg * ref_t).max()
    g.adjoint_record(0)


def test_checkpoint_interval_does_not_change_gradient(small):
    m, om, g, info = small
    cell = cell_grid_2x2x2(om)
    grads = []
    for every in (3, 50, 100000):
        g.adjoint_record(every)
        out = _run(m, g)
        if not grads:
            d_obs, mask = adjoint_misfit_case(out.fields)
            dJ9 = mask * (out.fields - d_obs)
        gc, gt, tm = g.adjoint(dJ9, cell, 8)
        grads.append(gc)
        assert tm["blocks"] >= 1 and tm["factors"] >= 1
    g.adjoint_record(0)
    for q in grads[1:]:
        assert np.abs(q - grads[0]).max() <= 1e-9 * np.abs(grads[0]).max()


@pytest.mark.parametrize("legacy", [False, True])
def test_adjoint_matches_finite_differences(small, legacy):
    m, om, g, info = small
    cell = cell_grid_2x2x2(om)
    g.adjoint_record(50)
    out = _run(m, g, legacy_linux=legacy)
    d_obs, mask = adjoint_misfit_case(out.fields)
    dJ9 = mask * (out.fields - d_obs)
    gc, _, _ = g.adjoint(dJ9, cell, 8)
    g.adjoint_record(0)    # the finite-difference runs below record nothing
    forced = out.trial_accepted.astype(np.int32)
    h = 1e-3
    sig0, mu0 = info["sig"], info["mu"]
    try:
        for c in (0, 5):
            Js = []
            for sgn in (1, -1):
                sig = sig0.copy()
                sig[cell == c] *= np.exp(sgn * h)
                g.set_media(sig, mu0)
                g.assemble()
                r = _run(m, g, legacy_linux=legacy, forced=forced)
                Js.append(0.5 * float(np.sum(mask * (r.fields - d_obs) ** 2)))
            fd = (Js[0] - Js[1]) / (2 * h)
            assert abs(gc[c] - fd) <= 1e-4 * abs(fd), (c, gc[c], fd)
    finally:
        g.set_media(sig0, mu0)
        g.assemble()


def test_adjoint_refuses_unrecorded_and_turn_off_runs(small):
    m, om, g, info = small
    g.adjoint_record(0)
    _run(m, g, max_steps=30)
    with pytest.raises(RuntimeError):
        g.adjoint(np.zeros((1, 1, 9)))
    g.set_sources([(info["src_edg"], info["src_drc"])], m.ctl.source_type, 3, m.ctl.t0, m.ctl.current)
    try:
        g.adjoint_record(10)
        with pytest.raises(RuntimeError):
            _run(m, g, max_steps=30)
    finally:
        g.adjoint_record(0)
        g.set_sources([(info["src_edg"], info["src_drc"])], m.ctl.source_type, m.ctl.pulse_type, m.ctl.t0,
                      m.ctl.current)


def test_lognormal_cell_model_gradient_matches_finite_differences_on_32_cells():
    """The config-3 workload at reduced size: the 3-D block model with its 64
    line receivers, log-normal cell conductivities (median 0.01 S/m, 0.5
    decades) on the 32 x 32 x 16 grid of 25 x 25 x 12.5 m cells, observations
    of a seeded 0.1-decade perturbation at 40 gates, J = 1/2 sum of squared
    dBz/dt gate residuals.  The adjoint gradient against central differences
    (log sigma +- 1e-3, decisions replayed) on 32 random cells of the grid:
    1e-4 relative, plus 1e-6 of the largest cell gradient for cells whose
    gradient is small (their difference quotient carries the rounding of J)."""
    import bench
    from temf3dt_b200 import inversion, synth
    kw = dict(bench.COMMON)
    kw.update(h_core=200.0, h_z=60.0, ratio=2.5, time_maximum=2e-4)
    m = synth.build_model("block", seed=3, **kw)
    md = bench.config3_media(m)
    gates = np.logspace(-6, np.log10(1.9e-4), 40)
    args = (m.ctl.sp_division, m.ctl.sp_double, m.ctl.sp_dblesize, m.ctl.time_maximum)
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        g.set_media(md["sig_true"], md["mu"])
        g.assemble()
        o = g.run(*args)
        d_obs = inversion.gate_matrix(o.times, gates) @ o.fields[:, :, 5]
        assert o.fields.shape[1] == 64
        g.set_media(md["sig"], md["mu"])
        g.assemble()
        g.adjoint_record(50)
        o = g.run(*args)
        J, dJ = inversion.dbdt_misfit(o.fields, o.times, gates, d_obs)
        grad, _, _ = g.adjoint(dJ, md["cell"], md["ncell"])
        g.adjoint_record(0)
        assert J > 0 and np.isfinite(grad).all()
        forced = o.trial_accepted.astype(np.int32)
        hit = np.unique(md["cell"][md["cell"] >= 0])
        pick = np.random.default_rng(32).choice(hit, size=32, replace=False)
        h = 1e-3
        scale = np.abs(grad).max()
        for k in pick:
            Jpm = []
            for sgn in (1.0, -1.0):
                sig = md["sig"].copy()
                sig[md["cell"] == k] *= np.exp(sgn * h)
                g.set_media(sig, md["mu"])
                g.assemble()
                r = g.run(*args, forced=forced)
                assert np.array_equal(r.steps, o.steps)
                Jpm.append(inversion.dbdt_misfit(r.fields, r.times, gates, d_obs)[0])
            fd = (Jpm[0] - Jpm[1]) / (2 * h)
            assert abs(grad[k] - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (int(k), grad[k], fd)
