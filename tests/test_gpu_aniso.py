"""Anisotropic media and the first-order absorbing boundary on the GPU
against the oracle (f_kind_ani, e_kind_ani, surface_integral,
src/FETD_FWD.f90:853-1007).  Marked ``gpu``; run on a B200."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fetd_oracle as O
from temf3dt_b200 import fetd
from tests.golden_cases import aniso_controls, oracle_model_with, tiny_synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    m = tiny_synth(time_maximum=1e-5)
    hc, oc = aniso_controls(m, bound_cond=1)
    om = oracle_model_with(m, oc)
    g = fetd.FetdGPU(0)
    info = fetd.load_case(g, m.mesh, hc)
    yield m, hc, om, g, info
    g.close()


def _csr(ia, ja, va, n):
    return sp.csr_matrix((va, ja - 1, ia - 1), shape=(n, n))


def test_anisotropic_absorbing_assembly_matches_oracle(case):
    m, hc, om, g, info = case
    for which, ref in ((0, om.B), (1, om.C)):
        G = _csr(*g.get_matrix(which), om.n)
        assert G.nnz == ref.nnz
        D = (G - ref).tocoo()
        R = ref.tocsr()
        rv = np.abs(np.asarray(R[D.row, D.col]).ravel())
        # entrywise: the absorbing term makes boundary entries ~1e12 times the interior ones
        assert (np.abs(D.data) <= 1e-11 * rv + 1e-15 * abs(ref).max()).all()


def test_anisotropic_absorbing_time_loop_matches_oracle(case):
    m, hc, om, g, info = case
    ref = O.run_fetd(om)
    c = m.ctl
    out = g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum,
                forced=np.array(ref.trial_accepted, dtype=np.int32))
    assert np.array_equal(out.steps, np.array(ref.steps))
    a, b = out.fields[:, 0, 3:6], ref.fields[:, 0, 3:6]
    assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max()


def test_adjoint_refuses_anisotropic_media(case):
    m, hc, om, g, info = case
    c = m.ctl
    g.adjoint_record(5)
    try:
        out = g.run(c.sp_division, c.sp_double, c.sp_dblesize, c.time_maximum, max_steps=12)
        with pytest.raises(RuntimeError):
            g.adjoint(np.zeros_like(out.fields))
    finally:
        g.adjoint_record(0)
