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
