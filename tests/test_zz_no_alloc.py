"""The allocation-free solve (temf_solve_noalloc) against the regular solve.

temf_solve_noalloc is for callers that cannot let the library call cudaMalloc
where they solve (a fixed device-memory budget, an allocator owned by the
application, another thread capturing CUDA work); its scratch is a static
device array.  This file is collected last so that a run stopping at the first
failure has run every other test already; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import fetd_oracle as O
from temf3dt_b200 import fetd
from tests.golden_cases import small_synth, synth_oracle_model

pytestmark = pytest.mark.gpu

# same criterion as the other solve tests: backward error <= 1e-12 of ||b||
BACKWARD_TOL = 1e-12


def test_noalloc_solve_matches_regular_solve_twice():
    import torch

    m = small_synth()
    om = synth_oracle_model(m)
    dt = 1e-6
    A = 3 * O.full_from_upper(om.B) + 2 * dt * O.full_from_upper(om.C)
    rng = np.random.default_rng(11)
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        assert g.factor(1, dt) == 0
        for call in range(2):          # two calls in a row share the static scratch
            b = A @ rng.standard_normal(om.n)
            x_ref = g.solve(1, b)      # the existing entry point (host arrays)
            b_dev = torch.tensor(b, dtype=torch.float64, device="cuda")
            x_dev = torch.full_like(b_dev, float("nan"))
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            rc = g._L.temf_solve_noalloc(g._h, 1, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()))
            assert rc == 0, g.last_error()
            if call == 1:
                # the second call finds everything in place: the device's free
                # memory is what it was (cudaMemGetInfo, whole device)
                assert torch.cuda.mem_get_info()[0] == free_before
            x = x_dev.cpu().numpy()
            nb = np.linalg.norm(b)
            assert np.linalg.norm(A @ x - b) <= BACKWARD_TOL * nb
            assert np.linalg.norm(A @ x_ref - b) <= BACKWARD_TOL * nb
            # the two solutions agree through A to the same tolerance
            assert np.linalg.norm(A @ (x - x_ref)) <= 2 * BACKWARD_TOL * nb
        # an invalid slot is rejected with a status, not a fault
        assert g._L.temf_solve_noalloc(g._h, 2, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr())) != 0
