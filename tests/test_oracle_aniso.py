"""CPU checks of the anisotropic-media and first-order-ABC restatement
(f_kind_ani, e_kind_ani, surface_integral, src/FETD_FWD.f90:853-1007) and of
the host readers for them."""
import math
import os
import tempfile

import numpy as np

from oracle import fetd_oracle as O
from temf3dt_b200 import meshio
from tests.golden_cases import aniso_controls, oracle_model_with, synth_oracle_model, tiny_synth


def test_isotropic_tensors_reproduce_the_isotropic_integrals():
    m = tiny_synth()
    om = synth_oracle_model(m)
    a, b, c, d, vol, tl = O.geometry(om.nod_cor, om.tet_vex)
    S = np.eye(3)[None] * om.sig[:, None, None]
    F1, F2 = O.f_kind_iso(b, c, d, vol, tl, om.sig), O.f_kind_ani(b, c, d, vol, tl, S)
    assert np.abs(F1 - F2).max() <= 1e-14 * np.abs(F1).max()
    Tm = np.eye(3)[None] / om.mag[:, None, None]
    E1, E2 = O.e_kind_iso(b, c, d, vol, tl, 1.0 / om.mag), O.e_kind_ani(b, c, d, vol, tl, Tm)
    assert np.abs(E1 - E2).max() <= 1e-14 * np.abs(E1).max()


def test_rotation_keeps_the_reference_z_factor():
    # dz puts cos(angle 2) at (2,2) (src/FETD_FWD.f90:389): with angles (0, 0, 30)
    # that entry is 1, not cos(30)
    R = O.rotation([0.0, 0.0, math.radians(30.0)])
    assert R[1, 1] == 1.0 and abs(R[0, 0] - math.cos(math.radians(30.0))) < 1e-15
    for ang in ([10.0, 20.0, 30.0], [0.0, 45.0, 0.0], [5.0, 0.0, 60.0]):
        assert np.allclose(meshio.rotation(ang), O.rotation(np.radians(ang)), rtol=0, atol=1e-15)


def test_boundary_faces_and_absorbing_term():
    m = tiny_synth()
    om = synth_oracle_model(m)
    faces = O.boundary_faces(om.nod_cor, om.tet_vex)
    assert faces.sum() > 0
    lo, hi = om.nod_cor.min(axis=0), om.nod_cor.max(axis=0)
    for t, f in zip(*np.nonzero(faces)):
        P = om.nod_cor[om.tet_vex[t, O.IND_TRI[f]] - 1]
        # every boundary face lies in one face plane of the box
        assert any(np.all(P[:, k] == lo[k]) or np.all(P[:, k] == hi[k]) for k in range(3))
    W = O.surface_integral(om.nod_cor, om.tet_vex, faces)
    assert np.abs(W - W.transpose(0, 2, 1)).max() <= 1e-14 * np.abs(W).max()
    assert np.count_nonzero(np.abs(W).sum(axis=(1, 2))) == np.count_nonzero(faces.any(axis=1))


def test_anisotropic_control_file_round_trip():
    m = tiny_synth()
    hc, oc = aniso_controls(m)
    path = os.path.join(tempfile.mkdtemp(), "aniso.cntl")
    meshio.write_cntl(path, hc)
    txt = open(path).read()
    assert "anisotropic:" in txt
    back = meshio.read_cntl(path)
    assert back.aniso_domains == hc.aniso_domains and back.bound_cond == 1
    oc2 = O.read_cntl(path)
    assert oc2.aniso and np.allclose(oc2.sig_ani, oc.sig_ani) and np.allclose(oc2.sig_ang, oc.sig_ang)
    sig9, mu9 = meshio.media_tensors_per_tet(m.mesh.tet_phy, back)
    om = oracle_model_with(m, oc2)
    earth = np.flatnonzero(m.mesh.tet_phy == back.aniso_domains[1][0])[0]
    assert np.allclose(sig9[earth].reshape(3, 3), O.media_tensor(oc.sig_ani[1], oc.sig_ang[1]))
    assert om.B.nnz > 0


def test_oracle_runs_with_anisotropy_and_absorbing_boundary():
    m = tiny_synth(time_maximum=5e-6)
    hc, oc = aniso_controls(m)
    res = O.run_fetd(oracle_model_with(m, oc))
    iso = O.run_fetd(synth_oracle_model(m))
    assert np.isfinite(res.fields).all()
    assert np.abs(res.fields[:, 0, 5] - iso.fields[:, 0, 5]).max() > 1e-3 * np.abs(iso.fields[:, 0, 5]).max()
