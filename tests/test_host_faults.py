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
