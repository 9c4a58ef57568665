"""Parity at the bench's full size: the first time steps of the 1.48M-edge
block model on the GPU against the oracle's adaptive loop on the CPU
supernodal Cholesky (an independent factor/solve on the host cores, same
ordering), receiver by receiver."""
import os
import sys

import numpy as np
import pytest

from oracle import fetd_oracle as O
from oracle import supernodal_cpu as SN
from temf3dt_b200 import fetd
from tests.golden_cases import ROOT, synth_oracle_model

pytestmark = pytest.mark.gpu

STEPS = 12


def test_block_model_first_steps_match_the_cpu_restatement():
    sys.path.insert(0, ROOT)
    import bench
    m = bench.model_for(1)
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        out = g.run(m.ctl.sp_division, m.ctl.sp_double, m.ctl.sp_dblesize, m.ctl.time_maximum, max_steps=STEPS)
    SN.build()
    om = synth_oracle_model(m)
    ref = O.run_fetd(om, max_steps=STEPS, slots=SN.SupernodalSlots(om))
    assert np.array_equal(out.steps, np.array(ref.steps))
    for lo in (0, 3):                               # E, then dB/dt: relative to the largest value of the group
        a, b = out.fields[:, :, lo:lo + 3], ref.fields[:, :, lo:lo + 3]
        scale = np.abs(b).max() + 1e-300
        err = (np.abs(a - b) / scale).max()
        assert err <= 1e-8, (lo, err)
