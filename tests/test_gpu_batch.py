"""Several independent layered models stepped together (temf_batch_*): each
model's output equals its own single-model run, with the merged solve
kernels, CUDA graphs and the autotuner in play.  Marked ``gpu``; run on a
B200."""
import numpy as np
import pytest

from temf3dt_b200 import fetd, synth

pytestmark = pytest.mark.gpu

# uneven mesh sizes (about 85k to 135k tets)
CASES = [(0, 0.25), (1, 0.3), (2, 0.2), (3, 0.35)]


@pytest.fixture(scope="module")
def models():
    out = []
    for seed, sc in CASES:
        m = synth.build_model("layered", seed=seed, scale=sc, ratio=2.0, time_maximum=2e-4, sp_double=40)
        g = fetd.FetdGPU(0)
        fetd.load_case(g, m.mesh, m.ctl)
        out.append((m, g))
    yield out
    for _, g in out:
        g.close()


def _args(m):
    c = m.ctl
    return c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_matches_single_runs(models, graphs):
    singles = [g.run(*_args(m)) for m, g in models]
    with fetd.FetdBatch([g for _, g in models]) as b:
        outs = b.run(*_args(models[0][0]), graphs=graphs, autotune=True)
        tm = b.timing()
        tu = b.tuning()
    assert tu["tuned"] and tm["merged_solves"] > 0 and tm["steps"] > 0
    assert len([x for x in tu["candidate_ms"] if x > 0]) == 6
    for s, o in zip(singles, outs):
        if not np.array_equal(s.trial_accepted, o.trial_accepted):
            continue  # a trial error within rounding of 1e-4 may flip; the schedules then differ
        assert np.array_equal(s.steps, o.steps)
        assert np.array_equal(s.times, o.times)
        ref = s.fields[:, :, :6]
        assert np.abs(o.fields[:, :, :6] - ref).max() <= 1e-9 * np.abs(ref).max()
    same = sum(np.array_equal(s.trial_accepted, o.trial_accepted) for s, o in zip(singles, outs))
    assert same >= len(models) - 1


def test_batch_step_limit_and_preset_tuning(models):
    # a preset schedule (level-aligned merge, all resident CTAs) and a step limit
    with fetd.FetdBatch([g for _, g in models]) as b:
        b.set_tuning(1, 100)
        outs = b.run(*_args(models[0][0]), max_steps=90)
        tu = b.tuning()
    assert tu["order"] == 1 and tu["grid_pct"] == 100
    single = models[1][1].run(*_args(models[1][0]), max_steps=90)
    o = outs[1]
    if np.array_equal(single.trial_accepted, o.trial_accepted):
        assert np.array_equal(single.steps, o.steps)
        ref = single.fields[:, :, :6]
        assert np.abs(o.fields[:, :, :6] - ref).max() <= 1e-9 * np.abs(ref).max()


def test_batch_rejects_bad_input(models):
    m, g = models[0]
    with pytest.raises(RuntimeError):
        fetd.FetdBatch([g, g])


def test_batch_members_match_the_oracle():
    """Three small models of two kinds and uneven size (14.5k, 19.6k and
    23.2k edges) stepped as one batch: every member keeps the oracle's own
    adaptive schedule (adap_euler, src/FETD_FWD.f90:1229-1464, run on that
    model alone), and its receiver E and dB/dt agree with the oracle to 1e-8
    of each trace's maximum, B to 1e-8 of its maximum."""
    from oracle import fetd_oracle as O
    from tests.golden_cases import synth_oracle_model, tiny_synth
    ms = [tiny_synth(), tiny_synth(h_core=150, radius=250.0),
          synth.build_model("layered", seed=1, scale=0.08, ratio=3.0, sp_double=8, sp_division=4,
                            time_maximum=2e-5)]
    refs = [O.run_fetd(synth_oracle_model(m)) for m in ms]
    gs = []
    try:
        for m in ms:
            g = fetd.FetdGPU(0)
            gs.append(g)
            fetd.load_case(g, m.mesh, m.ctl)
        with fetd.FetdBatch(gs) as b:
            outs = b.run(*_args(ms[0]), autotune=True)
            assert b.timing()["merged_solves"] > 0
    finally:
        for g in gs:
            g.close()
    for o, r in zip(outs, refs):
        assert np.array_equal(o.trial_accepted, np.array(r.trial_accepted))
        assert np.array_equal(o.steps, np.array(r.steps))
        ref = r.fields
        scale = np.abs(ref[:, :, :6]).max(axis=0)
        assert (np.abs(o.fields[:, :, :6] - ref[:, :, :6]) / np.maximum(scale, 1e-300)).max() <= 1e-8
        assert np.abs(o.fields[:, :, 6:] - ref[:, :, 6:]).max() <= 1e-8 * np.abs(ref[:, :, 6:]).max()
