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
