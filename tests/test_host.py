"""Host-side logic of the package and the C ABI that runs without a GPU:
exported symbols, mesh topology, ordering/symbolic analysis, file formats and
the synthetic model generator."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import fetd_oracle as O
from temf3dt_b200 import _lib, fetd, meshio, synth
from tests.golden_cases import ROOT, fixture_mesh, host_control, load_fixture, tiny_synth


def _header_functions():
    with open(os.path.join(ROOT, "include", "temf_b200.h")) as fh:
        txt = fh.read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(temf_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    lib = _lib.lib()
    names = _header_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, "no ctypes signature for %s" % n
    assert b"sm_100a" in lib.temf_version()


def test_topology_matches_oracle():
    fx = load_fixture("src_small_mod_small")
    tv = fx["tet_vex"].astype(np.int64)
    ev, te, td = fetd.mesh_topology(tv)
    e2, t2, d2 = O.build_topology(tv)
    assert np.array_equal(ev, e2) and np.array_equal(te, t2) and np.array_equal(td, d2)


def test_source_edges_follow_reference_convention():
    fx = load_fixture("linux_mod_big")
    ev, _, _ = fetd.mesh_topology(fx["tet_vex"])
    se, sd = fetd.source_edges(ev, fx["src_vex"])
    oe, od = O.source_edges(ev, fx["src_vex"].astype(np.int64))
    assert np.array_equal(se, oe) and np.array_equal(sd, od)
    assert sd[-1] == -1 and (sd[:-1] == 1).all()


def _grid_pattern(nx, ny, nz):
    """7-point pattern of an nx*ny*nz grid with coordinates."""
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    rows, cols = [], []
    for ax, sh in ((2, 1), (1, 1), (0, 1)):
        a = np.take(idx, np.arange(idx.shape[ax] - 1), axis=ax).ravel()
        b = np.take(idx, np.arange(1, idx.shape[ax]), axis=ax).ravel()
        rows += [a, b]; cols += [b, a]
    rows = np.concatenate(rows); cols = np.concatenate(cols)
    n = nx * ny * nz
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    xadj = np.zeros(n + 1, dtype=np.int64)
    np.add.at(xadj, rows + 1, 1)
    xadj = np.cumsum(xadj)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    xyz = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    return n, xadj, cols.astype(np.int32), xyz


def _symbolic(n, xadj, adj, xyz):
    perm = np.zeros(n, dtype=np.int32)
    st = np.zeros(9)
    xa = np.ascontiguousarray(xadj, dtype=np.int64)
    rc = _lib.lib().temf_symbolic_host(n, xa.ctypes.data_as(C.POINTER(C.c_longlong)), _lib.iptr(adj),
                                       _lib.dptr(np.ascontiguousarray(xyz)), _lib.iptr(perm), _lib.dptr(st))
    assert rc == 0
    return perm, st


def test_symbolic_nnz_matches_dense_cholesky():
    """The column counts of the symbolic factorisation equal the nonzero count
    of a dense Cholesky of a random SPD matrix with the same pattern in the
    computed order (no numerical cancellation in practice); the supernodes
    (with amalgamation zeros) hold at least that many."""
    n, xadj, adj, xyz = _grid_pattern(9, 8, 7)
    perm, st = _symbolic(n, xadj, adj, xyz)
    assert np.array_equal(np.sort(perm), np.arange(n))
    rng = np.random.default_rng(3)
    A = np.zeros((n, n))
    for i in range(n):
        for p in range(xadj[i], xadj[i + 1]):
            A[i, adj[p]] = -rng.uniform(0.1, 1.0)
    A = A + A.T
    A[np.arange(n), np.arange(n)] = np.abs(A).sum(axis=1) + 1.0
    L = np.linalg.cholesky(A[np.ix_(perm, perm)])
    assert int((np.abs(L) > 0).sum()) == int(st[8])
    assert st[3] >= st[8]
    assert st[1] >= 1 and st[2] >= 1
    # flops are at least the dense-column count lower bound
    assert st[5] > st[3]


def test_symbolic_on_reference_mesh():
    fx = load_fixture("src_small_mod_small")
    ev, te, _ = fetd.mesh_topology(fx["tet_vex"])
    n = len(ev)
    import scipy.sparse as sp
    r = np.repeat(te - 1, 6, axis=1).ravel(); c = np.tile(te - 1, (1, 6)).ravel()
    G = sp.coo_matrix((np.ones(len(r)), (r, c)), shape=(n, n)).tocsr()
    G.setdiag(0); G.eliminate_zeros(); G.sort_indices()
    xyz = 0.5 * (fx["nod_cor"][ev[:, 0] - 1] + fx["nod_cor"][ev[:, 1] - 1])
    perm, st = _symbolic(n, G.indptr.astype(np.int64), G.indices.astype(np.int32), xyz)
    assert np.array_equal(np.sort(perm), np.arange(n))
    assert st[3] < 0.05 * n * n       # far from dense
    assert st[3] >= (G.nnz // 2 + n)  # at least the lower triangle of A


def test_meshio_roundtrip(tmp_path):
    m = tiny_synth()
    p = str(tmp_path / "m.mesh")
    meshio.write_mesh(p, m.mesh)
    r = meshio.read_mesh(p)
    assert np.array_equal(r.tet_vex, m.mesh.tet_vex) and np.allclose(r.nod_cor, m.mesh.nod_cor, rtol=0, atol=0)
    assert np.array_equal(r.src_vex, m.mesh.src_vex)
    # the oracle's own reader agrees
    o = O.read_mesh(p)
    assert np.array_equal(o["tet_vex"], m.mesh.tet_vex) and np.array_equal(o["src_vex"], m.mesh.src_vex)
    pc = str(tmp_path / "m.cntl")
    meshio.write_cntl(pc, m.ctl)
    c2 = meshio.read_cntl(pc)
    oc = O.read_cntl(pc)
    assert c2.sp_double == m.ctl.sp_double and np.allclose(c2.rec_cor, m.ctl.rec_cor)
    assert oc.step_dble == m.ctl.sp_double and np.allclose(oc.time_channels, m.ctl.time_points)


def test_read_reference_cntl():
    for name in ("linux_mod_big", "src_small_mod_small"):
        c = host_control(load_fixture(name))
        assert c.sp_mthd == 2 and c.sp_dblesize == 2 and c.output[5] and c.output.sum() == 1
        assert c.domains[0][0] == 11 and c.domains[0][1] > 0


def test_field_roundtrip(tmp_path):
    steps = np.arange(4)
    times = np.array([0.0, 1e-8, 2e-8, 3.5e-8])
    f = np.random.default_rng(0).standard_normal((4, 2, 9))
    mask = np.zeros(9, dtype=bool); mask[[3, 5]] = True
    p = str(tmp_path / "x.field")
    meshio.write_field(p, steps, times, f, mask)
    r = meshio.read_field(p)
    assert r.shape == (4, 2 + 2 * 2)
    # Fortran E15.5 keeps 5 significant digits
    assert np.allclose(r[:, 2:].reshape(4, 2, 2), f[:, :, [3, 5]], rtol=6e-5, atol=0)


@pytest.mark.parametrize("kind", ["halfspace", "multiloop", "layered"])
def test_synth_models(kind):
    kw = {"halfspace": dict(h_core=250, ratio=2.5, h_z=50, z_core=150),
          "multiloop": dict(n_loops=3, h_core=60, ratio=2.2, h_z=60, scale=1.0),
          "layered": dict(scale=0.2, ratio=2.5, seed=4)}[kind]
    m = synth.build_model(kind, **kw)
    P = m.mesh.nod_cor[m.mesh.tet_vex - 1]
    d = np.einsum("ti,ti->t", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))
    assert (d > 0).all()
    if kind == "layered":
        # 3-6 layers with conductivities in [1e-4, 1e-1] S/m under air
        sig = [dom[1] for dom in m.ctl.domains[1:]]
        assert 3 <= len(sig) <= 6 and all(1e-4 <= v <= 1e-1 for v in sig)
        assert set(np.unique(m.mesh.tet_phy)) <= {dom[0] for dom in m.ctl.domains}
    ev, _, _ = fetd.mesh_topology(m.mesh.tet_vex)
    cols = m.source_columns(ev)
    se, sd = fetd.source_edges(ev, m.mesh.src_vex)
    assert np.array_equal(cols[0][0], se) and np.array_equal(cols[0][1], sd)
    for lp in m.loops:   # closed loop: consecutive vertices are mesh edges
        assert len(lp) >= 4
    # every receiver lies strictly inside exactly one tet
    for p in m.receivers:
        X = m.mesh.nod_cor[m.mesh.tet_vex - 1]
        mid = X.mean(axis=1)
        near = np.nonzero(np.linalg.norm(mid - p, axis=1) < 5000)[0]
        inside = 0
        for t in near:
            T = np.concatenate([X[t], np.ones((4, 1))], axis=1)
            lam = np.linalg.solve(T.T, np.append(p, 1.0))
            if (lam > 1e-9).all():
                inside += 1
        assert inside == 1


def _edge_pattern(model):
    """Edge-adjacency pattern (no diagonal) and edge midpoints of a synthetic mesh."""
    import scipy.sparse as sp
    from temf3dt_b200 import fetd
    ev, te, _ = fetd.mesh_topology(model.mesh.tet_vex)
    n, T = ev.shape[0], te.shape[0]
    I = sp.csr_matrix((np.ones(6 * T), (np.repeat(np.arange(T), 6), (te - 1).reshape(-1))), shape=(T, n))
    A = (I.T @ I).tocsr()
    A.setdiag(0)
    A.eliminate_zeros()
    A.sort_indices()
    mid = 0.5 * (model.mesh.nod_cor[ev[:, 0] - 1] + model.mesh.nod_cor[ev[:, 1] - 1])
    return n, A.indptr.astype(np.int64), A.indices.astype(np.int32), np.ascontiguousarray(mid)


@pytest.mark.parametrize("kind", ["grid", "mesh"])
def test_solve_schedules_replay(kind):
    """The persistent sweeps' task schedules, replayed on the host for both
    chunk heights: claimed in order every wait targets an earlier task, and
    through the ready queue every task is handed out once, after its inputs."""
    if kind == "grid":
        n, xadj, adj, xyz = _grid_pattern(13, 11, 9)
    else:
        from tests.golden_cases import tiny_synth
        n, xadj, adj, xyz = _edge_pattern(tiny_synth())
    msg = C.create_string_buffer(256)
    rc = _lib.lib().temf_schedule_check(n, xadj.ctypes.data_as(C.POINTER(C.c_longlong)), _lib.iptr(adj),
                                        _lib.dptr(xyz), msg, 256)
    assert rc == 0, msg.value.decode()


def test_ordering_does_not_depend_on_host_threads(monkeypatch):
    """The nested-dissection halves and the three axis evaluations of large
    subsets run on separate host threads; the permutation and the symbolic
    statistics are the same for one thread and for several."""
    n, xadj, adj, xyz = _grid_pattern(64, 60, 56)   # 215k unknowns: both threading thresholds reached
    out = {}
    for t in ("1", "3", "8"):
        monkeypatch.setenv("TEMF_HOST_THREADS", t)
        out[t] = _symbolic(n, xadj, adj, xyz)
    for t in ("3", "8"):
        assert np.array_equal(out[t][0], out["1"][0])
        assert np.array_equal(out[t][1][[0, 1, 2, 3, 4, 5, 8]], out["1"][1][[0, 1, 2, 3, 4, 5, 8]])


def test_topology_on_renumbered_mesh_matches_oracle():
    """Edge numbering, tet->edge map and signs of the library (counting sort
    by the smaller vertex) against the oracle's restatement, on a synthetic
    mesh whose vertices are renumbered and whose tets are shuffled, so that
    vertex indices and tet order carry no structure."""
    m = tiny_synth()
    rng = np.random.default_rng(11)
    nv = m.mesh.nod_cor.shape[0]
    relabel = rng.permutation(nv) + 1
    tv = relabel[m.mesh.tet_vex - 1][rng.permutation(m.mesh.tet_vex.shape[0])]
    ev, te, td = fetd.mesh_topology(tv)
    e2, t2, d2 = O.build_topology(tv.astype(np.int64))
    assert np.array_equal(ev, e2) and np.array_equal(te, t2) and np.array_equal(td, d2)


def test_fortran_interfaces_cover_the_header():
    """The ISO_C_BINDING module include/temf_b200.f90 declares every entry
    point of include/temf_b200.h with the same number of arguments, bound to
    the same C name."""
    with open(os.path.join(ROOT, "include", "temf_b200.h")) as fh:
        txt = re.sub(r"/\*.*?\*/", "", fh.read(), flags=re.S)
    header = {}
    for m in re.finditer(r"\b(temf_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
        args = m.group(2).strip()
        header[m.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    with open(os.path.join(ROOT, "include", "temf_b200.f90")) as fh:
        src = fh.read().replace("&\n", " ")
    fortran = {m.group(1): (0 if not m.group(2).strip() else len(m.group(2).split(",")))
               for m in re.finditer(r"function (temf_[a-z0-9_]+)\(([^)]*)\)", src)}
    bound = dict(re.findall(r"function (temf_[a-z0-9_]+)\([^)]*\)\s*bind\(C, name=\"([a-z0-9_]+)\"\)", src))
    assert set(header) <= set(fortran), sorted(set(header) - set(fortran))
    for name, n in header.items():
        assert fortran[name] == n, name
        assert bound.get(name) == name, name
    # the status codes match the header's
    with open(os.path.join(ROOT, "include", "temf_b200.h")) as fh:
        codes = dict(re.findall(r"#define (TEMF_E[A-Z]+|TEMF_OK) \(?(-?\d+)\)?", fh.read()))
    for k, v in codes.items():
        assert re.search(r"\b%s = %s\b" % (k, re.escape(v)), src), k


def test_fortran_pardiso_shim_keeps_the_reference_argument_lists():
    """include/pardiso_temf.f90 is a module named pardiso_multi_real_mpi with
    the reference's five public subroutines and their argument lists
    (src/FETD_UTILITY.f90:833-837,861,879,938,959,977), so adap_euler's calls
    compile unchanged; each forwards to the matching temf_pardiso_* entry."""
    with open(os.path.join(ROOT, "include", "pardiso_temf.f90")) as fh:
        src = re.sub(r"&\s*\n\s*", " ", re.sub(r"!.*", "", fh.read()))
    assert re.search(r"^module pardiso_multi_real_mpi\b", src, flags=re.M)
    want = {"pardiso_alloc": ["max_matrix"],
            "pardiso_direct_1": ["num_m", "symm", "n_in", "nnz_in", "ia", "ja", "va", "log"],
            "pardiso_direct_2": ["num_m", "b_in", "x_out", "ia", "ja", "va"],
            "pardiso_direct_3": ["num_m"],
            "pardiso_dealloc": []}
    subs = {m.group(1): [a.strip() for a in m.group(2).split(",") if a.strip()] if m.group(2) is not None else []
            for m in re.finditer(r"^\s*subroutine (pardiso_[a-z0-9_]+)(?:\(([^)]*)\))?", src, flags=re.M)}
    for name, args in want.items():
        assert subs.get(name) == args, (name, subs.get(name))
        body = src.split("subroutine %s" % name, 1)[1].split("end subroutine %s" % name, 1)[0]
        assert "temf_" + name in body, name
    public = re.search(r"public ::([^\n]*)", src).group(1)
    for name in want:
        assert name in public, name
    # optional log argument, as in the reference
    assert re.search(r"logical, optional, intent\(in\) :: log", src)


@pytest.mark.parametrize("case", ["single", "disconnected", "isolated_and_chain", "coincident_points"])
def test_analysis_of_degenerate_patterns(case):
    """Ordering, symbolic analysis and the schedule replay on patterns a mesh
    can degenerate to: one unknown, no edges, isolated unknowns beside a
    chain, and unknowns that all sit at one point (no axis can split them)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(1)
    n, rows, cols, xyz = {
        "single": (1, [], [], np.zeros((1, 3))),
        "disconnected": (40, [], [], rng.random((40, 3))),
        "isolated_and_chain": (500, list(range(100)), list(range(1, 101)), rng.random((500, 3))),
        "coincident_points": (300, rng.integers(0, 300, 2000), rng.integers(0, 300, 2000), np.zeros((300, 3))),
    }[case]
    A = sp.coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n)).tocsr()
    A = ((A + A.T) > 0).astype(float).tocsr()
    A.setdiag(0)
    A.eliminate_zeros()
    A.sort_indices()
    xadj, adj = A.indptr.astype(np.int64), A.indices.astype(np.int32)
    perm, st = _symbolic(n, xadj, adj, np.ascontiguousarray(xyz))
    assert np.array_equal(np.sort(perm), np.arange(n)) and st[8] >= n
    msg = C.create_string_buffer(256)
    rc = _lib.lib().temf_schedule_check(n, xadj.ctypes.data_as(C.POINTER(C.c_longlong)), _lib.iptr(adj),
                                        _lib.dptr(np.ascontiguousarray(xyz)), msg, 256)
    assert rc == 0, msg.value.decode()


def test_single_tet_topology_follows_ind_tet():
    """Local edges (1,2),(1,3),(1,4),(2,3),(4,2),(3,4) of ind_tet
    (src/FETD_FWD.f90:23): the fifth runs from vertex 4 to 2, against the
    global (2,4) edge, so its sign is -1."""
    ev, te, td = fetd.mesh_topology(np.array([[1, 2, 3, 4]]))
    assert ev.tolist() == [[1, 2], [1, 3], [1, 4], [2, 3], [2, 4], [3, 4]]
    assert te.tolist() == [[1, 2, 3, 4, 5, 6]] and td.tolist() == [[1, 1, 1, 1, -1, 1]]


def test_gate_matrix_follows_the_field2_interpolation():
    """inversion.gate_matrix reproduces the .field2 gates (interp_lin between
    the rows that bracket each gate, src/FETD_FWD.f90:1625-1640 and
    src/FETD_UTILITY.f90:21-31), and dbdt_misfit's derivative matches a
    finite difference of its misfit."""
    from temf3dt_b200 import inversion
    rng = np.random.default_rng(4)
    times = np.concatenate([[0.0], np.cumsum(rng.uniform(1e-7, 3e-6, 60))])
    f = rng.standard_normal((len(times), 3, 9))
    gates = np.sort(rng.uniform(1e-6, times[-1] * 0.99, 12))
    W = inversion.gate_matrix(times, gates)
    for g, tg in enumerate(gates):
        i = int(np.argmax(times >= tg))
        want = O.interp_lin(times[i - 1], f[i - 1], times[i], f[i], tg)
        assert np.allclose(np.tensordot(W[g], f, axes=1), want, rtol=1e-12, atol=1e-12)
    assert (W[:, :].sum(axis=1) == pytest.approx(1.0))
    late = inversion.gate_matrix(times, [times[-1] * 2])
    assert not late.any()
    d_obs = rng.standard_normal((len(gates), 3))
    J, dJ = inversion.dbdt_misfit(f, times, gates, d_obs)
    k = (17, 1, 5)
    h = 1e-6
    f2 = f.copy()
    f2[k] += h
    J2, _ = inversion.dbdt_misfit(f2, times, gates, d_obs)
    assert abs((J2 - J) / h - dJ[k]) <= 1e-5 * max(1.0, abs(dJ[k]))
    assert not dJ[:, :, :5].any() and not dJ[:, :, 6:].any()


def test_inversion_grid_cells():
    """Tet -> cell map by centroid on a regular grid (x slowest, z fastest),
    -1 outside, and the per-cell conductivity it carries."""
    from temf3dt_b200 import inversion
    grid = inversion.InversionGrid((4, 3, 2), ((0.0, 4.0), (0.0, 3.0), (0.0, 2.0)))
    pts = np.array([[0.5, 0.5, 0.5], [3.5, 2.5, 1.5], [1.2, 0.1, 1.9], [-0.1, 1.0, 1.0], [1.0, 1.0, 2.5]])
    assert grid.cell_of_points(pts).tolist() == [0, 23, 7, -1, -1]
    sc = inversion.lognormal_cells(grid.ncell, 0.01, 0.5, 3)
    assert np.allclose(np.median(np.log10(inversion.lognormal_cells(20000, 0.01, 0.5, 3))), -2.0, atol=0.02)
    sig = inversion.sigma_with_cells(np.full(5, 1e-12), grid.cell_of_points(pts), sc)
    assert sig[0] == sc[0] and sig[1] == sc[23] and sig[3] == 1e-12
