"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle
and the reference's shipped outputs.  Marked ``gpu``; run on a B200.

Tolerances (FP64 throughout):
  * assembled matrices, receiver operators: 1e-13 of the largest entry
    (different summation order / cofactor expansion only);
  * solves: backward error ||A x - b|| / ||b|| <= 1e-12;
  * receiver dB/dt of a time loop vs the oracle on the same mesh and schedule:
    1e-8 relative to the trace maximum (different orderings of an
    ill-conditioned FP64 factorisation; the target is 1e-6);
  * vs the reference's .field files: their print precision (6e-5 for the
    5-digit src_small file, 6e-4 for the 4-digit LINUX files).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fetd_oracle as O
from temf3dt_b200 import fetd
from tests.golden_cases import (host_model_from_fixture, load_fixture, oracle_model_from_fixture, small_synth,
                                synth_oracle_model, tiny_synth)

pytestmark = pytest.mark.gpu

TRACE_RTOL = 1e-8


@pytest.fixture(scope="module")
def small():
    m = small_synth()
    om = synth_oracle_model(m)
    g = fetd.FetdGPU(0)
    info = fetd.load_case(g, m.mesh, m.ctl)
    yield m, om, g, info
    g.close()


def _csr(ia, ja, va, n):
    return sp.csr_matrix((va, ja - 1, ia - 1), shape=(n, n))


def test_assembly_matches_oracle(small):
    m, om, g, info = small
    for which, ref in ((0, om.B), (1, om.C)):
        G = _csr(*g.get_matrix(which), om.n)
        assert G.nnz == ref.nnz
        assert abs(G - ref).max() <= 1e-13 * abs(ref).max()


def test_receiver_operators_and_location(small):
    m, om, g, info = small
    assert np.array_equal(info["rec_tet"], om.rec_tet)
    na, da = g.receiver_operators()
    assert np.abs(na - om.n_arr).max() <= 1e-13 * np.abs(om.n_arr).max()
    assert np.abs(da - om.d_arr).max() <= 1e-13 * np.abs(om.d_arr).max()
    # point location agrees with the oracle's scan, including "not found"
    pts = np.array([m.receivers[0], [1e6, 1e6, 1e6]])
    loc = g.locate(pts, 1e5)
    assert loc[0] == om.rec_tet[0] and loc[1] == 0


@pytest.mark.parametrize("dt", [1e-7, 1e-5, 1e-3])
def test_factor_solve_backward_error(small, dt):
    m, om, g, info = small
    A = 3 * O.full_from_upper(om.B) + 2 * dt * O.full_from_upper(om.C)
    assert g.factor(1, dt) == 0
    rng = np.random.default_rng(7)
    X0 = rng.standard_normal((om.n, 3))
    B = A @ X0
    X = g.solve(1, B)
    for k in range(3):
        assert np.linalg.norm(A @ X[:, k] - B[:, k]) <= 1e-12 * np.linalg.norm(B[:, k])
    # a single column through the same path: same backward error (the forward
    # sweep accumulates with FP64 atomics and A is ill-conditioned, so the two
    # solutions are not compared entry by entry)
    x = g.solve(1, B[:, 0])
    assert np.linalg.norm(A @ x - B[:, 0]) <= 1e-12 * np.linalg.norm(B[:, 0])


@pytest.mark.parametrize("nrhs", [1, 64])
def test_tuned_sweep_schedules_solve_to_backward_error(small, nrhs):
    """The autotuner times each candidate queue split and keeps one; solves
    with the chosen schedule keep backward error 1e-12 (1 and 64 columns)."""
    m, om, g, info = small
    dt = 1e-6
    A = 3 * O.full_from_upper(om.B) + 2 * dt * O.full_from_upper(om.C)
    assert g.factor(1, dt) == 0
    split, cand = g.tune_solve(1, nrhs)
    assert split in cand and len(cand) >= 2
    assert g.solve_schedule(nrhs) == (split, True)
    rng = np.random.default_rng(5)
    X0 = rng.standard_normal((om.n, nrhs))
    B = A @ X0
    X = g.solve(1, B if nrhs > 1 else B[:, 0]).reshape(om.n, nrhs)
    rel = np.linalg.norm(A @ X - B, axis=0) / np.linalg.norm(B, axis=0)
    assert rel.max() <= 1e-12, rel.max()


@pytest.mark.parametrize("level", [1, 2, 3, 5, 8])
def test_subtree_sweeps_solve_to_backward_error(small, level):
    """Single-column solves with the supernodes below `level` swept as whole
    subtrees (one warp each, no waits) before and after the persistent task
    sweeps, with and without the ready queue above them, and with and without
    run leaders (one CTA walking the column blocks of a wide supernode), and
    with every task above the subtrees in the queue: backward error 1e-12,
    and the same solution as the plan without subtrees to that tolerance."""
    m, om, g, info = small
    dt = 1e-6
    A = 3 * O.full_from_upper(om.B) + 2 * dt * O.full_from_upper(om.C)
    assert g.factor(1, dt) == 0
    L = min(level, int(g.stats()["levels"]) - 1)
    b = A @ np.random.default_rng(level).standard_normal(om.n)
    nb = np.linalg.norm(b)
    try:
        g.set_solve_plan(0, 0, run_leaders=False)
        x0 = g.solve(1, b)
        for split in (L, L + 3, int(g.stats()["levels"])):
            for leaders in (True, False):
                g.set_solve_plan(L, split, run_leaders=leaders)
                plan = g.solve_plan()
                assert plan["tree_level"] == L and plan["split"] == split and plan["n_trees"] > 0
                assert plan["run_leaders"] == leaders
                x = g.solve(1, b)
                assert np.linalg.norm(A @ x - b) <= 1e-12 * nb
                assert np.linalg.norm(A @ (x - x0)) <= 2e-12 * nb
    finally:
        g.tune_solve(1, 1)


def test_block_solve_of_many_columns(small):
    """70 right-hand sides: one full 64-column block through the tensor-core
    block sweeps plus a 6-column remainder; every column to backward error
    1e-12."""
    m, om, g, info = small
    dt = 1e-5
    A = 3 * O.full_from_upper(om.B) + 2 * dt * O.full_from_upper(om.C)
    assert g.factor(2, dt) == 0
    rng = np.random.default_rng(11)
    X0 = rng.standard_normal((om.n, 70))
    B = A @ X0
    X = g.solve(2, B)
    R = A @ X - B
    rel = np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)
    assert rel.max() <= 1e-12, rel.max()


def test_spmv_matches_oracle(small):
    m, om, g, info = small
    x = np.random.default_rng(1).standard_normal(om.n)
    for which, ref in ((0, om.B), (1, om.C)):
        y = g.spmv(which, x)
        r = O.full_from_upper(ref) @ x
        assert np.linalg.norm(y - r) <= 1e-13 * np.linalg.norm(r)


def test_time_loop_matches_oracle(small):
    """Full adaptive BDF2 run (9 trials, accepts and rejects) vs the oracle."""
    m, om, g, info = small
    res = O.run_fetd(om)
    out = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum)
    assert np.array_equal(out.steps, np.array(res.steps))
    assert np.array_equal(out.times, np.array(res.times))
    assert np.array_equal(out.trial_accepted, np.array(res.trial_accepted))
    assert np.allclose(out.trial_errors, res.trial_errors, rtol=1e-5)
    ref = res.fields
    scale = np.abs(ref[:, :, :6]).max(axis=0)
    err = np.abs(out.fields[:, :, :6] - ref[:, :, :6]) / np.maximum(scale, 1e-300)
    assert err.max() <= TRACE_RTOL, err.max()
    # B is the rectangle-rule integral of dB/dt (src/FETD_FWD.f90:1612-1620)
    assert np.allclose(out.fields[:, :, 6:], ref[:, :, 6:], rtol=0, atol=TRACE_RTOL * np.abs(ref[:, :, 6:]).max())
    # gates (.field2) follow the same interpolation
    gates = np.logspace(-6.5, np.log10(m.ctl.time_maximum * 0.9), 7)
    gv, done = g.gates(gates)
    assert done.all()
    k = np.searchsorted(np.array(res.times), gates)
    for q, t in enumerate(gates):
        i = k[q]
        expect = O.interp_lin(res.times[i - 1], ref[i - 1], res.times[i], ref[i], t)
        assert np.allclose(gv[q], expect, rtol=0, atol=TRACE_RTOL * np.abs(ref).max())


def test_graph_and_eager_paths_agree(small):
    m, om, g, info = small
    a = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum, graphs=True)
    b = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum, graphs=False)
    assert np.array_equal(a.steps, b.steps)
    # the solves are deterministic; the factor's scatter uses FP64 atomics, so
    # two runs agree to rounding, not bitwise
    assert np.allclose(a.fields, b.fields, rtol=0, atol=1e-10 * np.abs(a.fields).max())


def test_forced_schedule_replay(small):
    m, om, g, info = small
    a = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum)
    forced = np.where(a.trial_accepted, 0, 1)          # invert every decision
    b = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum, forced=forced)
    n = len(a.trial_accepted)      # the inverted schedule reaches t_max with more trials
    assert np.array_equal(b.trial_accepted[:n], ~a.trial_accepted)


def test_src_small_example_matches_reference_field():
    """The reference's src_small example on the GPU vs its shipped .field
    (5 digits) and vs the oracle fixture replayed with the same decisions."""
    fx = load_fixture("src_small_mod_small")
    mesh, ctl, scale = host_model_from_fixture(fx, sigma_rescale=True)
    z = np.load("tests/golden/oracle_src_small.npz")
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, mesh, ctl)
        out = g.run(ctl.sp_division, ctl.sp_double, ctl.sp_dblesize, ctl.time_maximum, max_steps=len(z["steps"]) - 1)
        gold = fx["field"]
        n = 630
        assert np.array_equal(out.steps[:n], gold[:n, 0].astype(int))
        v = out.fields[:n, 0, 5] * scale
        rel = np.abs(v[1:] - gold[1:n, 2]) / np.abs(gold[1:n, 2])
        assert rel.max() < 6e-5, rel.max()
        # vs the oracle with identical decisions (the trial errors sit near 1e-4 at late time)
        nt = len(z["trial_accepted"])
        rep = g.run(ctl.sp_division, ctl.sp_double, ctl.sp_dblesize, ctl.time_maximum,
                    forced=z["trial_accepted"].astype(np.int32), max_steps=len(z["steps"]) - 1)
        assert np.array_equal(rep.steps, z["steps"][:len(rep.steps)])
        ref = z["fields"][:len(rep.steps), 0, 5]
        err = np.abs(rep.fields[:, 0, 5] - ref) / np.abs(ref).max()
        assert err.max() <= TRACE_RTOL, err.max()


@pytest.mark.parametrize("name", ["linux_mod_big", "linux_mod_small"])
def test_linux_examples_match_reference_field(name):
    """The reference's LINUX examples (108k edges, 918/922 rows to t = 0.1 s)
    on the GPU with the schedule rule of the build that wrote them, against
    the shipped .field (4 printed digits), every row.

    1. With the file's own accept/reject decisions (read off its time
       column; the committed oracle run replays them): every row's step and
       time, and dB_z/dt to the print.
    2. The free run decides by itself.  Its dB_z/dt matches to the print up
       to the first row whose time differs, and a difference may only come
       from a trial that FP64 solver rounding can decide either way: the
       late trials' error estimates are dominated by the air fields, which the
       1e-12 S/m air leaves nearly undetermined (the receiver dB/dt agree to
       1e-14 while those estimates differ between solvers by tens of percent),
       so the GPU's and the oracle's estimates must lie on both sides of 1e-4,
       or further apart than the oracle's estimate is from it -- or the
       restated rule on the oracle's estimate (file history) must itself
       decide differently from the file there, as at trial 19 of
       mod_small."""
    from tests.golden_cases import GOLDEN, golden_field_report
    fx = load_fixture(name)
    z = np.load(os.path.join(GOLDEN, "oracle_" + name + ".npz"))
    mesh, ctl, _ = host_model_from_fixture(fx)
    gold = fx["field"]
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, mesh, ctl)
        rep = g.run(ctl.sp_division, ctl.sp_double, ctl.sp_dblesize, ctl.time_maximum, legacy_linux=True,
                    forced=z["trial_accepted"].astype(np.int32))
        out = g.run(ctl.sp_division, ctl.sp_double, ctl.sp_dblesize, ctl.time_maximum, legacy_linux=True)
    first, _, rel = golden_field_report(rep.steps, rep.times, rep.fields[:, 0, 5], [], gold, ctl.sp_double)
    assert len(rep.steps) == len(gold) and first == len(gold), (len(rep.steps), first)
    assert np.array_equal(rep.steps, gold[:, 0].astype(int))
    assert rel < 6e-4, rel
    # the early trials (earth fields dominate the estimate) agree with the oracle's to 1e-3
    early = np.abs(rep.trial_errors[:10] / z["trial_errors"][:10] - 1.0)
    assert early.max() < 1e-3, early
    first, decided, rel = golden_field_report(out.steps, out.times, out.fields[:, 0, 5], out.trial_errors, gold,
                                              ctl.sp_double)
    print("%s: free run rows %d / %d, first differing row %d, its trial error %s, dBz/dt rel %.2e"
          % (name, len(out.steps), len(gold), first, decided, rel))
    assert rel < 6e-4, rel
    if first < len(gold) or len(out.steps) != len(gold):
        from tests.golden_cases import free_divergence_explained, golden_decisions
        k = int(out.steps[min(first, len(out.steps) - 1)]) // ctl.sp_double - 1
        assert decided is not None
        assert free_divergence_explained(k, decided, z["trial_errors"], golden_decisions(gold, ctl.sp_double)), \
            (k, decided, float(z["trial_errors"][k]))


def test_multi_rhs_columns_match_single_runs():
    """Three loops as three RHS columns of one run == three single runs."""
    m = tiny_synth()
    with fetd.FetdGPU(0) as g:
        info = fetd.load_case(g, m.mesh, m.ctl)
        se, sd = info["src_edg"], info["src_drc"]
        cols = [(se, sd), (se[: len(se) // 2], sd[: len(sd) // 2]), (se[::-1], -sd[::-1])]
        singles = []
        for c in cols:
            g.set_sources([c], 1, 1, m.ctl.t0, 1.0)
            g.set_receivers(info["rec_tet"], m.ctl.rec_cor)
            singles.append(g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum))
        # the batched run shares one schedule: replay the first column's decisions
        g.set_sources(cols, 1, 1, m.ctl.t0, 1.0)
        g.set_receivers(np.repeat(info["rec_tet"], 3), np.repeat(m.ctl.rec_cor, 3, axis=0), rec_rhs=[0, 1, 2])
        forced = singles[0].trial_accepted.astype(np.int32)
        b = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum, forced=forced)
    for k in (0, 1, 2):
        s = singles[k]
        if not np.array_equal(s.trial_accepted, singles[0].trial_accepted):
            continue
        assert np.allclose(b.fields[:, k, :6], s.fields[:, 0, :6], rtol=0, atol=1e-10 * np.abs(s.fields[:, 0, :6]).max())
    # column 2 is column 0 reversed in sign: fields are negated
    assert np.allclose(b.fields[:, 2, 3:6], -b.fields[:, 0, 3:6], rtol=1e-9, atol=1e-12 * np.abs(b.fields[:, 0, 3:6]).max())


@pytest.mark.parametrize("pulse", [2, 3])
def test_pulse_types_match_oracle(pulse):
    """Impulse (type 2) and step-off with the DC pass first (type 3)."""
    m = tiny_synth(pulse_type=pulse)
    om = synth_oracle_model(m)
    res = O.run_fetd(om)
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        out = g.run(m.ctl.sp_division, m.ctl.sp_double, 2, m.ctl.time_maximum,
                    forced=np.array(res.trial_accepted, dtype=np.int32))
    assert np.array_equal(out.steps, np.array(res.steps))
    ref = res.fields[:, :, :6]
    err = np.abs(out.fields[:, :, :6] - ref) / np.abs(ref).max(axis=0)
    assert err.max() <= TRACE_RTOL, err.max()


def test_pardiso_shim_and_pivot_status(small):
    """pardiso_direct_1/2/3 on the user's 1-based upper CSR; a non-SPD matrix
    gives a positive status (first failing column), not a trap, and the
    context stays usable."""
    m, om, g, info = small
    dt = 1e-6
    A = (3 * om.B + 2 * dt * om.C).tocsr()
    A.sort_indices()
    ia, ja, va = A.indptr + 1, A.indices + 1, A.data.copy()
    g.pardiso_alloc(2)
    assert g.pardiso_direct_1(1, ia, ja, va) == 0
    Af = O.full_from_upper(A)
    b = Af @ np.random.default_rng(2).standard_normal(om.n)
    x = g.pardiso_direct_2(1, b)
    assert np.linalg.norm(Af @ x - b) <= 1e-12 * np.linalg.norm(b)
    bad = va.copy()
    diag = np.nonzero(ja - 1 == np.repeat(np.arange(om.n), np.diff(A.indptr)))[0]
    bad[diag[5]] = -abs(bad[diag[5]])
    st = g.pardiso_direct_1(2, ia, ja, bad)
    assert st > 0
    # the first slot is still valid and usable
    x2 = g.pardiso_direct_2(1, b)
    assert np.linalg.norm(Af @ x2 - b) <= 1e-12 * np.linalg.norm(b)
    g.pardiso_direct_3(1)
    g.pardiso_dealloc()


@pytest.mark.parametrize("case", ["one_negative_pivot", "shifted"])
def test_pardiso_indefinite_fallback(small, case):
    """A matrix that is not positive definite: pardiso_direct_1 reports the
    first non-positive pivot (the reference's warning before it retries with
    mtype -2, src/FETD_UTILITY.f90:923-935) and factors it in the indefinite
    mode (L S L^T, S = diag(+-1), static pivot perturbation); pardiso_direct_2
    with two refinement steps solves it to backward error 1e-10 and agrees
    with SuperLU (pivoting LU) on the same matrix.  Cases: one planted
    negative diagonal entry, and 3 M - 2 dt K with dt = 2e-6 (many negative
    eigenvalues).  The other slot and the next SPD factorisation stay usable."""
    import scipy.sparse.linalg as spla
    m, om, g, info = small
    if case == "one_negative_pivot":
        A = (3 * om.B + 2 * 1e-6 * om.C).tocsr()
    else:
        A = (3 * om.B - 2 * 2e-6 * om.C).tocsr()
    A.sort_indices()
    ia, ja, va = A.indptr + 1, A.indices + 1, A.data.copy()
    if case == "one_negative_pivot":
        diag = np.nonzero(ja - 1 == np.repeat(np.arange(om.n), np.diff(A.indptr)))[0]
        va[diag[17]] = -abs(va[diag[17]])
    Au = sp.csr_matrix((va, ja - 1, ia - 1), shape=(om.n, om.n))
    Af = O.full_from_upper(Au)
    g.pardiso_alloc(2)
    try:
        st = g.pardiso_direct_1(2, ia, ja, va)
        assert st > 0
        rng = np.random.default_rng(23)
        b = Af @ rng.standard_normal(om.n)
        x = g.pardiso_direct_2(2, b)
        nb = np.linalg.norm(b)
        assert np.linalg.norm(Af @ x - b) <= 1e-10 * nb
        ref = spla.splu(Af.tocsc()).solve(b)
        assert np.linalg.norm(Af @ (x - ref)) <= 2e-10 * nb
        # an SPD matrix in the other slot, then again in this one
        As = (3 * om.B + 2 * 1e-6 * om.C).tocsr()
        As.sort_indices()
        for slot in (1, 2):
            assert g.pardiso_direct_1(slot, As.indptr + 1, As.indices + 1, As.data) == 0
            Asf = O.full_from_upper(As)
            y = g.pardiso_direct_2(slot, Asf @ np.ones(om.n))
            assert np.linalg.norm(Asf @ y - Asf @ np.ones(om.n)) <= 1e-12 * np.linalg.norm(Asf @ np.ones(om.n))
    finally:
        g.pardiso_dealloc()


def test_halfspace_central_loop_matches_analytic_response():
    """dBz/dt at the centre of a 500 m loop on a 0.001 S/m half-space against
    the closed-form response (Ward & Hohmann eq. 4.98) convolved with the erf
    step-on waveform: within 2 % over 1e-5..1e-3 s.  The staircase loop's
    enclosed area sets the effective radius; 10 m cells below the surface."""
    from temf3dt_b200 import synth
    from tests.halfspace import erf_step_on_dbzdt
    m = synth.build_model("halfspace", h_core=50, ratio=1.6, h_z=10, z_core=300, time_maximum=2e-3)
    sv = m.mesh.src_vex - 1
    P = m.mesh.nod_cor[sv[:, 0]]
    area = 0.5 * abs(np.sum(P[:, 0] * np.roll(P[:, 1], -1) - np.roll(P[:, 0], -1) * P[:, 1]))
    a_eff = np.sqrt(area / np.pi)
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        g.run(m.ctl.sp_division, m.ctl.sp_double, m.ctl.sp_dblesize, m.ctl.time_maximum)
        gates = np.logspace(-5, -3, 21)
        v, done = g.gates(gates)
    assert done.all()
    ana = erf_step_on_dbzdt(gates, 1e-3, a_eff, m.ctl.t0)
    rel = np.abs(v[:, 0, 5] - ana) / np.abs(ana)
    assert rel.max() <= 0.02, rel


def test_device_wait_timeout_is_reported_and_the_context_recovers(small):
    """A device wait that can never be met (one input more expected than any
    task provides) gives up after the context's spin limit: the kernel
    finishes, temf_solve reports the timeout, and the next solve on the same
    context is correct (failure detection without a GPU fault)."""
    m, om, g, info = small
    dt = 1e-6
    A = 3 * O.full_from_upper(om.B) + 2 * dt * O.full_from_upper(om.C)
    assert g.factor(1, dt) == 0
    b = A @ np.random.default_rng(9).standard_normal(om.n)
    try:
        for split in (0, int(g.stats()["levels"])):   # the wait claimed in order, then the queue slot
            g.set_solve_plan(2, split)
            g.set_wait_limit(1 << 12, inject_unmet_wait=True)
            with pytest.raises(RuntimeError, match="timed out"):
                g.solve(1, b)
            g.set_wait_limit(0)
            x = g.solve(1, b)
            assert np.linalg.norm(A @ x - b) <= 1e-12 * np.linalg.norm(b)
    finally:
        g.set_wait_limit(0)
        g.tune_solve(1, 1)
