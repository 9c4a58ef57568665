"""CPU checks of the oracle adjoint: the fields -> samples chain rule, the
graph replay of the forward run, and the gradient against central finite
differences (decisions held fixed)."""
import numpy as np
import pytest

from oracle import fetd_adjoint as AD
from oracle import fetd_oracle as O
from tests.golden_cases import adjoint_misfit_case, cell_grid_2x2x2, synth_oracle_model, tiny_synth


def _fields_from_samples(s, steps, dts):
    """solution_output's 9 columns from the 6 raw samples per row."""
    f = np.zeros(s.shape[:2] + (9,))
    f[:, :, :3] = s[:, :, :3]
    f[:, :, 3:6] = s[:, :, 3:6] * (np.asarray(steps) != 0)[:, None, None]
    f[:, :, 6:9] = np.cumsum(f[:, :, 3:6] * np.asarray(dts)[:, None, None], axis=0)
    return f


def test_fields_grad_chain_rule():
    rng = np.random.default_rng(3)
    R, nrec = 17, 3
    steps = np.arange(R)
    dts = rng.uniform(1e-7, 1e-6, R)
    s = rng.standard_normal((R, nrec, 6))
    d = rng.standard_normal((R, nrec, 6))
    g9 = rng.standard_normal((R, nrec, 9))
    lhs = np.sum(g9 * (_fields_from_samples(s + d, steps, dts) - _fields_from_samples(s, steps, dts)))
    rhs = np.sum(AD.fields_grad_to_samples(g9, steps, dts) * d)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


@pytest.fixture(scope="module")
def tiny_case():
    om = synth_oracle_model(tiny_synth(time_maximum=1e-5))
    g, states, rows = AD.forward_graph(om)
    return om, g, states, rows


def _J(rows, d_obs, mask):
    return 0.5 * float(np.sum(mask * (rows - d_obs) ** 2))


@pytest.mark.parametrize("legacy", [False, True])
def test_graph_replays_the_forward_run(tiny_case, legacy):
    om = tiny_case[0]
    ref = O.run_fetd(om, legacy_linux=legacy)
    g, states, rows = AD.forward_graph(om, legacy_linux=legacy) if legacy else tiny_case[1:]
    assert rows.shape == ref.fields.shape
    assert np.abs(rows - ref.fields).max() <= 1e-12 * np.abs(ref.fields).max()
    assert g.decisions == list(ref.trial_accepted)
    assert len(g.row_node) == len(rows)
    assert np.array_equal(g.row_step, ref.steps)


def test_adjoint_matches_finite_differences(tiny_case):
    om, g, states, rows = tiny_case
    cell = cell_grid_2x2x2(om)
    d_obs, mask = adjoint_misfit_case(rows)
    dJ9 = mask * (rows - d_obs)
    dJ = AD.fields_grad_to_samples(dJ9, g.row_step, g.row_dt)
    grad = AD.adjoint_gradient(om, g, states, dJ, cell, 8)
    h = 1e-4
    for c in (0, 3, 5):
        Js = []
        for sgn in (1, -1):
            sig = om.sig.copy()
            sig[cell == c] *= np.exp(sgn * h)
            _, _, r2 = AD.forward_graph(AD.with_sigma(om, sig), decisions=g.decisions)
            Js.append(_J(r2, d_obs, mask))
        fd = (Js[0] - Js[1]) / (2 * h)
        # central differences: O(h^2) truncation plus rounding of J / h
        assert abs(grad[c] - fd) <= 1e-5 * abs(fd), (c, grad[c], fd)
