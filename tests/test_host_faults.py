"""Host-side fault handling without a GPU: malformed input files and wrong
arguments to the host-only entry points end in an error, never a crash."""
import ctypes as C

import numpy as np
import pytest

from oracle import fetd_oracle as O
from temf3dt_b200 import _lib, meshio
from tests.golden_cases import tiny_synth


def test_truncated_mesh_file_is_rejected(tmp_path):
    m = tiny_synth()
    p = tmp_path / "m.mesh"
    meshio.write_mesh(str(p), m.mesh)
    lines = p.read_text().splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.strip().startswith("Tetra"))
    (tmp_path / "cut.mesh").write_text("\n".join(lines[:k + 5]) + "\n")
    with pytest.raises(ValueError):
        meshio.read_mesh(str(tmp_path / "cut.mesh"))
    with pytest.raises(ValueError):
        O.read_mesh(str(tmp_path / "cut.mesh"))


def test_control_file_without_required_keys_is_rejected(tmp_path):
    m = tiny_synth()
    p = tmp_path / "c.cntl"
    meshio.write_cntl(str(p), m.ctl)
    text = p.read_text()
    (tmp_path / "nosrc.cntl").write_text(text.replace("source: 1", "sourcex: 1"))
    with pytest.raises(ValueError):
        meshio.read_cntl(str(tmp_path / "nosrc.cntl"))
    with pytest.raises(ValueError):
        O.read_cntl(str(tmp_path / "nosrc.cntl"))


def test_host_entry_points_return_error_codes():
    L = _lib.lib()
    m = tiny_synth()
    tv = np.asfortranarray(m.mesh.tet_vex.astype(np.int32))
    T = tv.shape[0]
    ne = C.c_int(0)
    assert L.temf_mesh_count_edges(T, _lib.iptr(tv), C.byref(ne)) == 0 and ne.value > 0
    ev = np.zeros(2 * ne.value, dtype=np.int32)
    te = np.zeros(6 * T, dtype=np.int32)
    td = np.zeros(6 * T, dtype=np.int32)
    # a wrong edge count is refused
    rc = L.temf_mesh_topology(T, _lib.iptr(tv), ne.value + 1, _lib.iptr(ev), _lib.iptr(te), _lib.iptr(td))
    assert rc < 0
    assert L.temf_mesh_topology(T, _lib.iptr(tv), ne.value, _lib.iptr(ev), _lib.iptr(te), _lib.iptr(td)) == 0
    # empty or NULL input to the host-only analysis
    assert L.temf_symbolic_host(0, None, None, None, None, None) < 0
    assert L.temf_schedule_check(0, None, None, None, None, 0) < 0


def _upper_csr_of_mesh():
    """1-based upper CSR of the edge-adjacency pattern (with the diagonal) of
    the small synthetic mesh: the structure adap_euler hands to
    pardiso_direct_1."""
    import scipy.sparse as sp
    from temf3dt_b200 import fetd
    m = tiny_synth()
    ev, te, _ = fetd.mesh_topology(m.mesh.tet_vex)
    n, T = ev.shape[0], te.shape[0]
    I = sp.csr_matrix((np.ones(6 * T), (np.repeat(np.arange(T), 6), (te - 1).reshape(-1))), shape=(T, n))
    A = sp.triu((I.T @ I).tocsr()).tocsr()
    A.sort_indices()
    return (A.indptr + 1).astype(np.int32), (A.indices + 1).astype(np.int32)


def test_pardiso_checker_accepts_the_step_pattern_and_rejects_planted_errors():
    from temf3dt_b200 import fetd
    ia, ja = _upper_csr_of_mesh()
    assert fetd.pardiso_checker(True, ia, ja) == (True, "")
    assert fetd.pardiso_checker(False, ia, ja)[0]
    r = 5                       # a row with several entries
    q0, q1 = ia[r] - 1, ia[r + 1] - 1
    assert q1 - q0 >= 3
    bad = ja.copy(); bad[q0 + 1], bad[q0 + 2] = bad[q0 + 2], bad[q0 + 1]
    ok, msg = fetd.pardiso_checker(True, ia, bad)
    assert not ok and "ascending" in msg and "row %d" % (r + 1) in msg
    bad = ja.copy(); bad[q0 + 2] = bad[q0 + 1]          # duplicate entry
    assert not fetd.pardiso_checker(True, ia, bad)[0]
    bad = ja.copy(); bad[q0] = r                         # (r+1, r) is below the diagonal
    ok, msg = fetd.pardiso_checker(True, ia, bad)
    assert not ok and "below the diagonal" in msg
    assert fetd.pardiso_checker(False, ia, bad)[0]       # a general matrix may hold it
    bad = ja.copy(); bad[-1] = len(ia)                   # column n + 1
    ok, msg = fetd.pardiso_checker(True, ia, bad)
    assert not ok and "out of range" in msg
    ok, msg = fetd.pardiso_checker(True, ia - 1, ja)     # zero-based row pointers
    assert not ok and "one-based" in msg
    ok, msg = fetd.pardiso_checker(True, ia, ja[:-1])    # nnz disagrees with ia(n+1)
    assert not ok and "nnz" in msg
    L = _lib.lib()
    ck = np.zeros(1, dtype=np.int32)
    assert L.temf_pardiso_checker(1, len(ia) - 1, len(ja), None, _lib.iptr(ja), _lib.iptr(ck), None, 0) < 0


def test_source_segment_that_is_not_a_mesh_edge_is_rejected():
    """A source segment must be an edge of the mesh (src_edg of model_ctl,
    src/FETD_FWD.f90:435-448); two opposite corners of a tet's neighbour are not."""
    from temf3dt_b200 import fetd
    m = tiny_synth()
    ev, _, _ = fetd.mesh_topology(m.mesh.tet_vex)
    se, sd = fetd.source_edges(ev, m.mesh.src_vex)
    assert len(se) == len(m.mesh.src_vex) and sd[-1] == -1
    edges = set(map(tuple, ev.tolist()))
    n = m.mesh.nod_cor.shape[0]
    bad = next((a, b) for a in range(1, n + 1) for b in range(a + 1, n + 1) if (a, b) not in edges)
    with pytest.raises(ValueError, match="not an edge"):
        fetd.source_edges(ev, np.array([bad]))
