"""`./FETD -f ROOT` end to end on the GPU: the C++ driver (temf_fetd, all
file handling in the library) against the Python driver (fetd.run_case) on
the same .mesh/.cntl files."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from temf3dt_b200 import fetd, meshio
from tests.golden_cases import ROOT, tiny_synth

pytestmark = pytest.mark.gpu


def _close(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a[:, 0], b[:, 0])                      # step / channel numbers
    scale = np.abs(b[:, 1:]).max(axis=0) + 1e-300
    assert (np.abs(a[:, 1:] - b[:, 1:]) <= 2e-5 * np.abs(b[:, 1:]) + 1e-9 * scale).all()


def test_native_driver_matches_python_driver(tmp_path):
    m = tiny_synth()
    a, b = str(tmp_path / "py"), str(tmp_path / "native")
    meshio.write_mesh(a + ".mesh", m.mesh)
    meshio.write_cntl(a + ".cntl", m.ctl)
    shutil.copy(a + ".mesh", b + ".mesh")
    shutil.copy(a + ".cntl", b + ".cntl")
    fetd.run_case(a)
    cli = os.path.join(ROOT, "temf3dt_b200", "temf_fetd")
    r = subprocess.run([cli, "-f", b], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    _close(meshio.read_field(b + ".field"), meshio.read_field(a + ".field"))
    _close(meshio.read_field(b + ".field2"), meshio.read_field(a + ".field2"))


def test_native_driver_reproduces_the_shipped_linux_field(tmp_path):
    """temf_fetd --legacy-linux on the reference's LINUX/mod_big_sig_0.001
    files (mesh re-emitted from the fixture, the shipped cntl text) against
    the shipped .field, as the Python path is checked in test_gpu_parity."""
    from tests.golden_cases import load_fixture
    fx = load_fixture("linux_mod_big")
    root = str(tmp_path / "mod_big")
    meshio.write_mesh(root + ".mesh", meshio.Mesh(fx["nod_cor"], fx["tet_vex"].astype(np.int64),
                                                  fx["tet_phy"].astype(np.int64), fx["src_vex"].astype(np.int64),
                                                  fx["src_phy"].astype(np.int64)))
    with open(root + ".cntl", "w") as fh:
        fh.write(str(fx["cntl"]))
    cli = os.path.join(ROOT, "temf3dt_b200", "temf_fetd")
    r = subprocess.run([cli, "-f", root, "--legacy-linux"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    out = meshio.read_field(root + ".field")
    gold = fx["field"]
    # the schedule may part from the file only at a trial that FP64 solver
    # rounding can decide either way (see test_linux_examples_match_reference_field):
    # there the GPU's estimate (from the same run through the Python driver,
    # the .field holds none) and the oracle's lie on both sides of 1e-4
    from tests.golden_cases import GOLDEN, golden_field_report, host_model_from_fixture
    z = np.load(os.path.join(GOLDEN, "oracle_linux_mod_big.npz"))
    mesh, ctl, _ = host_model_from_fixture(fx)
    first, _, rel = golden_field_report(out[:, 0].astype(int), out[:, 1], out[:, 2], [], gold, ctl.sp_double)
    assert rel < 6e-4, rel
    if first < len(gold) or len(out) != len(gold):
        with fetd.FetdGPU(0) as g:
            fetd.load_case(g, mesh, ctl)
            py = g.run(ctl.sp_division, ctl.sp_double, ctl.sp_dblesize, ctl.time_maximum, legacy_linux=True)
        from tests.golden_cases import free_divergence_explained, golden_decisions
        k = int(out[min(first, len(out) - 1), 0]) // ctl.sp_double - 1
        mine = float(py.trial_errors[k])
        assert free_divergence_explained(k, mine, z["trial_errors"], golden_decisions(gold, ctl.sp_double)), \
            (k, mine, float(z["trial_errors"][k]))


def test_mesh_field_snapshots_match_the_oracle():
    """vtkout snapshots (E, D, B at every tet centroid) of the GPU run against
    the oracle's vtk_field_save restatement, same trial decisions.

    E inside the air (1e-12 S/m) is not determined to 1e-8 by any of the
    solvers: its gradient part only meets the tiny air mass 3 M_air, so it
    carries the solve's rounding amplified by the air/earth contrast.  The
    oracle on SuperLU and the oracle on the CPU supernodal Cholesky (same
    FP64 loop, another elimination order) already differ there by 2.7e-8
    and 4e-7 of the group maximum at the two snapshots, while they agree to
    1e-14 on earth E, D and B.  So air E is held to ten times that measured
    solver-to-solver floor; everything else to 1e-9."""
    from oracle import fetd_oracle as O
    from oracle import supernodal_cpu as SN
    from tests.golden_cases import synth_oracle_model
    m = tiny_synth()
    times = [1e-6, 5e-6]
    om = synth_oracle_model(m)
    om.ctl.vtk_times = np.array(times)
    ref = O.run_fetd(om)
    SN.build()
    alt = O.run_fetd(om, slots=SN.SupernodalSlots(om, threads=2))
    assert alt.steps == ref.steps
    air = om.sig < 1e-6
    assert air.any() and (~air).any()
    with fetd.FetdGPU(0) as g:
        fetd.load_case(g, m.mesh, m.ctl)
        g.set_mesh_fields(times)
        out = g.run(m.ctl.sp_division, m.ctl.sp_double, m.ctl.sp_dblesize, m.ctl.time_maximum,
                    forced=np.array(ref.trial_accepted, dtype=np.int32))
        assert np.array_equal(out.steps, np.array(ref.steps))
        for i in range(len(times)):
            f, done = g.mesh_fields(i)
            assert done
            r, a = ref.mesh_fields[i], alt.mesh_fields[i]
            for lo in (0, 3, 6):
                scale = np.abs(r[:, lo:lo + 3]).max()
                err = np.abs(f[:, lo:lo + 3] - r[:, lo:lo + 3]).max(axis=1)
                if lo == 0:
                    floor = np.abs(a[air, 0:3] - r[air, 0:3]).max()
                    assert err[air].max() <= max(1e-8 * scale, 10.0 * floor), (i, err[air].max() / scale,
                                                                                floor / scale)
                    assert err[~air].max() <= 1e-9 * scale, (i, lo, err[~air].max() / scale)
                else:
                    assert err.max() <= 1e-9 * scale, (i, lo, err.max() / scale)


def test_native_driver_writes_the_msh_dumps(tmp_path):
    """temf_fetd with vtkout times and ROOT.msh present writes ROOT_i.msh;
    its element data match the oracle's msh_output to the 8 printed digits."""
    from oracle import fetd_oracle as O
    from tests.golden_cases import synth_oracle_model
    from tests.test_mesh_fields import _write_msh41
    m = tiny_synth()
    m.ctl.vtk_times = np.array([1e-6, 5e-6])
    m.ctl.output = np.array([1, 1, 1, 0, 0, 1, 0, 0, 1], dtype=bool)
    root = str(tmp_path / "v")
    meshio.write_mesh(root + ".mesh", m.mesh)
    meshio.write_cntl(root + ".cntl", m.ctl)
    _write_msh41(root + ".msh", m.mesh)
    cli = os.path.join(ROOT, "temf3dt_b200", "temf_fetd")
    r = subprocess.run([cli, "-f", root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    om = synth_oracle_model(m)
    om.ctl.vtk_times = m.ctl.vtk_times
    om.ctl.o_f = m.ctl.output
    ref = O.run_fetd(om)
    for i in (1, 2):
        O.write_msh_fields(root + ".msh", str(tmp_path / ("o_%d.msh" % i)), ref.mesh_fields[i - 1], m.ctl.output)

        def values(path):
            vals, on = [], False
            for ln in open(path):
                if ln.startswith("$ElementData"):
                    on, skip = True, 8
                    continue
                if ln.startswith("$EndElementData"):
                    on = False
                    continue
                if on:
                    if skip:
                        skip -= 1
                        continue
                    vals.append(float(ln.split()[1]))
            return np.array(vals)
        a, b = values(root + "_%d.msh" % i), values(str(tmp_path / ("o_%d.msh" % i)))
        assert a.shape == b.shape and len(a) == 5 * len(m.mesh.tet_vex)
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
