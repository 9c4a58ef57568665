"""The CPU supernodal Cholesky slots (the timed CPU baseline) against the
SuperLU slots of the oracle: backward error of the solves, the adaptive run
and the non-positive-pivot report.  CPU only."""
import numpy as np
import pytest

from oracle import fetd_oracle as O
from oracle import supernodal_cpu as SN
from tests.golden_cases import small_synth, synth_oracle_model, tiny_synth


@pytest.fixture(scope="module")
def small():
    SN.build()
    return synth_oracle_model(small_synth())


@pytest.mark.parametrize("threads", [1, 4])
def test_solves_are_backward_stable(small, threads):
    sl = SN.SupernodalSlots(small, threads=threads)
    rng = np.random.default_rng(3)
    for dt in (1e-7, 1e-5):
        sl.factor(1, dt)
        A = O.full_from_upper(3.0 * small.B + 2.0 * dt * small.C)
        x0 = rng.standard_normal(small.n)
        b = A @ x0
        x = sl.solve(1, b)
        assert np.linalg.norm(A @ x - b) <= 1e-12 * np.linalg.norm(b)


def test_adaptive_run_matches_superlu_slots():
    SN.build()
    om = synth_oracle_model(tiny_synth())
    ref = O.run_fetd(om)
    got = O.run_fetd(om, slots=SN.SupernodalSlots(om, threads=3))
    assert got.steps == ref.steps and got.trial_accepted == ref.trial_accepted
    scale = np.abs(ref.fields[:, :, :6]).max(axis=0)
    assert (np.abs(got.fields[:, :, :6] - ref.fields[:, :, :6]) <= 1e-7 * scale).all()


def test_non_positive_pivot_is_reported(small):
    sl = SN.SupernodalSlots(small, threads=2)
    with pytest.raises(np.linalg.LinAlgError):
        sl.factor(1, -1.0)     # 3 M - 2 K is indefinite
    sl.factor(2, 1e-6)         # the other slot is still usable
    b = np.ones(small.n)
    assert np.isfinite(sl.solve(2, b)).all()
