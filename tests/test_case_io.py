"""The library's C++ file front end (model_mesh, model_ctl, the .field
writer) against the Python readers and writer, on synthetic and on the
reference's shipped files (fixtures).  CPU only."""
import os

import numpy as np
import pytest

from temf3dt_b200 import fetd, meshio
from tests.golden_cases import aniso_controls, load_fixture, tiny_synth


def _write_case(tmp_path, mesh, ctl, name="case"):
    root = str(tmp_path / name)
    meshio.write_mesh(root + ".mesh", mesh)
    meshio.write_cntl(root + ".cntl", ctl)
    return root


def _same_control(cf, c):
    assert np.allclose(cf.rec_cor, c.rec_cor, rtol=0, atol=0)
    assert cf.rec_charac == c.rec_charac and cf.bound_cond == c.bound_cond
    assert (cf.source_type, cf.pulse_type, cf.t0, cf.current) == (c.source_type, c.pulse_type, c.t0, c.current)
    assert (cf.sp_mthd, cf.sp_division, cf.sp_double, cf.sp_dblesize) == \
        (c.sp_mthd, c.sp_division, c.sp_double, c.sp_dblesize)
    assert cf.time_maximum == c.time_maximum and np.array_equal(cf.output, c.output)
    if c.time_points is None:
        assert cf.time_points is None
    else:
        assert np.array_equal(cf.time_points, c.time_points)


def test_synthetic_case_reads_like_the_python_readers(tmp_path):
    m = tiny_synth()
    root = _write_case(tmp_path, m.mesh, m.ctl)
    cf = fetd.CaseFile(root)
    mesh = meshio.read_mesh(root + ".mesh")
    ctl = meshio.read_cntl(root + ".cntl")
    assert np.array_equal(cf.nod_cor, mesh.nod_cor) and np.array_equal(cf.tet_vex, mesh.tet_vex)
    assert np.array_equal(cf.tet_phy, mesh.tet_phy)
    assert np.array_equal(cf.src_vex, mesh.src_vex) and np.array_equal(cf.src_phy, mesh.src_phy)
    _same_control(cf, ctl)
    sig, mu, aniso = cf.media()
    s2, m2 = meshio.media_per_tet(mesh.tet_phy, ctl)
    assert not aniso and np.array_equal(sig, s2) and np.array_equal(mu, m2)


def test_anisotropic_media_match_the_python_tensors(tmp_path):
    m = tiny_synth()
    hc, _ = aniso_controls(m, bound_cond=1)
    root = _write_case(tmp_path, m.mesh, hc)
    cf = fetd.CaseFile(root)
    ctl = meshio.read_cntl(root + ".cntl")
    sig, mu, aniso = cf.media()
    s2, m2 = meshio.media_tensors_per_tet(m.mesh.tet_phy, ctl)
    assert aniso and cf.bound_cond == 1
    assert np.allclose(sig, s2, rtol=1e-15, atol=0) and np.allclose(mu, m2, rtol=1e-15, atol=0)


@pytest.mark.parametrize("name", ["linux_mod_big", "src_small_mod_small"])
def test_reference_files_read_like_the_fixtures(tmp_path, name):
    """The shipped mesh (re-emitted from the fixture arrays) and the shipped
    cntl text, read by the C++ front end."""
    fx = load_fixture(name)
    mesh = meshio.Mesh(fx["nod_cor"], fx["tet_vex"].astype(np.int64), fx["tet_phy"].astype(np.int64),
                       fx["src_vex"].astype(np.int64), fx["src_phy"].astype(np.int64))
    root = str(tmp_path / name)
    meshio.write_mesh(root + ".mesh", mesh)
    with open(root + ".cntl", "w") as fh:
        fh.write(str(fx["cntl"]))
    cf = fetd.CaseFile(root)
    assert np.array_equal(cf.nod_cor, fx["nod_cor"]) and np.array_equal(cf.tet_vex, fx["tet_vex"])
    assert np.array_equal(cf.src_vex, fx["src_vex"]) and np.array_equal(cf.tet_phy, fx["tet_phy"])
    _same_control(cf, meshio.read_cntl(root + ".cntl"))


def test_fortran_exponents_comments_and_errors(tmp_path):
    root = str(tmp_path / "f")
    with open(root + ".mesh", "w") as fh:
        fh.write(" MeshVersionFormatted 2\n Dimension\n 3\n Vertices\n 4\n"
                 " 0.0d0 0.0D0 0.0 1\n 1.5d+1 0 0 1\n 0 2.0E1 0 1\n 0 0 1.0d1 1\n"
                 " Tetrahedra\n 1\n 1 2 3 4 12\n End\n")
    with open(root + ".cntl", "w") as fh:
        fh.write("% comment\nreceivers: 1 ! one\n1.0d0 2.0 3.0\nrec_charac:\t5.0d0\nisotropic: 1\n12 1d-2 1 1\n"
                 "source: 1\n1 1 1.0d-6 1.0\nsp_mthd: 2\nsp_division: 10\ntime_maximum: 1.0d-3\n"
                 "sp_double: 20\nsp_dblesize: 2\noutput:\n0 0 0 0 0 1 0 0 0\nvtkout: 1\n1.0e-4\n")
    cf = fetd.CaseFile(root)
    assert np.array_equal(cf.nod_cor[1], [15.0, 0.0, 0.0]) and cf.nod_cor[3, 2] == 10.0
    assert cf.rec_charac == 5.0 and cf.t0 == 1e-6 and cf.time_maximum == 1e-3 and cf.vtkout == 1
    assert np.array_equal(cf.rec_cor[0], [1.0, 2.0, 3.0]) and cf.time_points is None
    # the completeness test of model_ctl
    with open(root + ".cntl", "w") as fh:
        fh.write("receivers: 1\n0 0 0\nisotropic: 1\n12 1 1 1\nsp_mthd: 2\n")
    with pytest.raises(ValueError, match="incomplete"):
        fetd.CaseFile(root)
    # a truncated mesh section
    with open(root + ".mesh", "w") as fh:
        fh.write(" Vertices\n 4\n 0 0 0 1\n")
    with pytest.raises(ValueError, match="truncated"):
        fetd.CaseFile(root)
    with pytest.raises(ValueError, match="cannot open"):
        fetd.CaseFile(str(tmp_path / "missing"))


def test_field_rows_are_written_like_the_python_writer(tmp_path):
    rng = np.random.default_rng(4)
    rows, nrec = 7, 3
    steps = np.arange(rows)
    times = np.concatenate([[0.0], np.cumsum(rng.uniform(1e-9, 1e-6, rows - 1))])
    fields = rng.standard_normal((rows, nrec, 9)) * 10.0 ** rng.integers(-14, 3, (rows, nrec, 9))
    fields[0] = 0.0
    fields[2, 1, 5] = -0.0
    for mask in ([0, 0, 0, 0, 0, 1, 0, 0, 0], [1, 1, 1, 1, 1, 1, 1, 1, 1], [1, 0, 0, 0, 1, 0, 0, 0, 1]):
        a, b = str(tmp_path / "a.field"), str(tmp_path / "b.field")
        fetd.write_field_rows(a, steps, times, fields, mask)
        meshio.write_field(b, steps, times, fields, np.array(mask, dtype=bool))
        with open(a) as fa, open(b) as fb:
            ta, tb = fa.read(), fb.read()
        assert ta == tb
        r = meshio.read_field(a)
        sel = np.nonzero(mask)[0]
        assert np.allclose(r[:, 2:].reshape(rows, nrec, len(sel)), fields[:, :, sel], rtol=1e-4, atol=0)
    first = open(a).readline()
    assert first.startswith("     0    0.00000E+00  ")


def test_command_line_driver_reports_usage_and_missing_files(tmp_path):
    import subprocess
    from tests.golden_cases import ROOT
    cli = os.path.join(ROOT, "temf3dt_b200", "temf_fetd")
    r = subprocess.run([cli], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([cli, "-f", str(tmp_path / "nothing")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_unknown_physical_domain_and_bad_writer_arguments(tmp_path):
    m = tiny_synth()
    ctl = meshio.read_cntl(_write_case(tmp_path, m.mesh, m.ctl) + ".cntl")
    ctl.domains = ctl.domains[:1]               # drop the earth domains
    root = _write_case(tmp_path, m.mesh, ctl, name="nodom")
    cf = fetd.CaseFile(root)
    with pytest.raises(ValueError, match="physical domain"):
        cf.media()
    from temf3dt_b200 import _lib
    L = _lib.lib()
    mask = np.ones(9, dtype=np.int32)
    assert L.temf_case_write_rows(None, 1, 1, None, None, None, _lib.iptr(mask)) < 0
    assert L.temf_case_write_rows(str(tmp_path / "x").encode(), 1, 1, None, None, None, _lib.iptr(mask)) < 0
    assert L.temf_case_write_rows(str(tmp_path / "x").encode(), 0, 0, None, None, None, _lib.iptr(mask)) == 0
    assert open(str(tmp_path / "x")).read() == ""
