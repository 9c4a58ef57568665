"""Whole-mesh field dumps (vtkout: vtk_field_save and msh_output,
src/FETD_FWD.f90:1642-1864), host parts: the library's per-tet centroid
fields and its Gmsh writer against the oracle's restatement.  CPU only."""
import numpy as np

from oracle import fetd_oracle as O
from temf3dt_b200 import fetd, meshio
from tests.golden_cases import synth_oracle_model, tiny_synth


def _write_msh41(path, mesh):
    """A Gmsh 4.1 file of a synthetic mesh: a line block (source edges)
    before the tetrahedra, whose tags start at 101."""
    N, T = len(mesh.nod_cor), len(mesh.tet_vex)
    with open(path, "w") as fh:
        fh.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        fh.write("$Nodes\n1 %d 1 %d\n3 1 0 %d\n" % (N, N, N))
        fh.write("".join("%d\n" % (k + 1) for k in range(N)))
        fh.write("".join("%.17g %.17g %.17g\n" % tuple(p) for p in mesh.nod_cor))
        fh.write("$EndNodes\n")
        S = len(mesh.src_vex)
        fh.write("$Elements\n2 %d 1 %d\n" % (S + T, 100 + T))
        fh.write("1 51 1 %d\n" % S)
        fh.write("".join("%d %d %d\n" % (k + 1, a, b) for k, (a, b) in enumerate(mesh.src_vex)))
        fh.write("3 1 4 %d\n" % T)
        fh.write("".join("%d %d %d %d %d\n" % ((101 + k,) + tuple(t)) for k, t in enumerate(mesh.tet_vex)))
        fh.write("$EndElements\n")


def test_centroid_fields_match_vtk_field_save():
    m = tiny_synth()
    om = synth_oracle_model(m)
    e = np.random.default_rng(2).standard_normal(om.n)
    mf = O.MeshFields(om)
    mf(2.5e-7, e)
    got = fetd.mesh_fields_host(om.nod_cor, om.tet_vex, om.tet_edg, om.tet_drc, e)
    for a, b in ((got[:, :3], mf.e), (got[:, 3:], mf.d)):
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()
    assert np.allclose(mf.b, mf.d * 2.5e-7, rtol=0, atol=0)


def test_vtk_snapshots_of_an_oracle_run():
    """The oracle's run keeps E, D, B at the first output row at or after
    each vtkout time; B is the D * dt sum over the rows up to it."""
    m = tiny_synth()
    om = synth_oracle_model(m)
    om.ctl.vtk_times = np.array([1e-6, 5e-6])
    res = O.run_fetd(om)
    assert sorted(res.mesh_fields) == [0, 1]
    f0, f1 = res.mesh_fields[0], res.mesh_fields[1]
    assert f0.shape == (len(om.tet_vex), 9) and np.abs(f1[:, 6:]).max() > 0
    assert not np.array_equal(f0, f1)


def test_msh_writer_matches_msh_output(tmp_path):
    m = tiny_synth()
    m.ctl.vtk_times = np.array([1e-6, 5e-6])
    m.ctl.output = np.array([1, 0, 1, 0, 0, 1, 0, 0, 1], dtype=bool)
    root = str(tmp_path / "case")
    meshio.write_mesh(root + ".mesh", m.mesh)
    meshio.write_cntl(root + ".cntl", m.ctl)
    _write_msh41(root + ".msh", m.mesh)
    cf = fetd.CaseFile(root)
    assert np.array_equal(cf.vtk_times, [1e-6, 5e-6])
    assert O.msh_tet_tags(root + ".msh") == list(range(101, 101 + len(m.mesh.tet_vex)))
    fields = np.random.default_rng(3).standard_normal((len(m.mesh.tet_vex), 9)) * 1e-7
    fields[0] = 0.0
    cf.write_msh(root + ".msh", str(tmp_path / "a_1.msh"), fields)
    O.write_msh_fields(root + ".msh", str(tmp_path / "b_1.msh"), fields, m.ctl.output)
    a = open(str(tmp_path / "a_1.msh")).read()
    b = open(str(tmp_path / "b_1.msh")).read()
    assert a == b
    assert a.count("$ElementData") == 4 and '"Ex data"' in a and '"Bz data"' in a
    line = next(ln for ln in a.splitlines() if ln.startswith("       102"))
    assert line.endswith(O._fortran_e(abs(fields[1, 0]), 16, 8))
    # a file whose tetrahedra do not match the mesh is refused
    with open(root + ".msh") as fh:
        txt = fh.read().replace("3 1 4 %d" % len(m.mesh.tet_vex), "3 1 4 %d" % (len(m.mesh.tet_vex) - 1))
    with open(str(tmp_path / "bad.msh"), "w") as fh:
        fh.write(txt)
    try:
        cf.write_msh(str(tmp_path / "bad.msh"), str(tmp_path / "c.msh"), fields)
        raise AssertionError("mismatched .msh accepted")
    except ValueError as err:
        assert "tetrahedra" in str(err)
