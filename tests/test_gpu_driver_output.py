"""The host driver's output options on a short run (fp64, CUDA-graph steps):

* --vtk-binary writes the reference's output.vtk data set as legacy VTK
  BINARY: the same dimensions, points and fields as the default ASCII file
  (to the ASCII file's 7 significant digits);
* --plot3d writes output.xyz / output.q in binary Plot3D: the input grid and
  the final conservative state, equal bit for bit to the grid file and the
  checkpoint's interior;
* --bc characteristic runs the characteristic far-field mode: the checkpoint
  matches the library's own run of that mode.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cbns3d_cuda_b200 import BC_CHARACTERISTIC, cases
from tests.helpers import per_var_rel_linf
from tests.test_gpu_parity import pair

pytestmark = pytest.mark.gpu

EXE = Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "bin" / "cbns3d_b200"


def _run(d, *opts):
    r = subprocess.run([str(EXE), "--quiet", "--graph", "--inviscid", *opts], cwd=d, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_binary_vtk_and_plot3d(tmp_path):
    c = cases.case_vortex(20, 14, 10)
    da = c.write(tmp_path / "ascii", nsteps=5, checkpoint_freq=5)
    db = c.write(tmp_path / "binary", nsteps=5, checkpoint_freq=5)
    _run(da)
    _run(db, "--vtk-binary", "--plot3d")
    assert (db / "output.vtk").read_bytes().split(b"\n")[2] == b"BINARY"
    dims_a, pts_a, f_a = cases.read_vtk(da / "output.vtk")
    dims_b, pts_b, f_b = cases.read_vtk(db / "output.vtk")
    assert dims_a == dims_b == c.shape and sorted(f_a) == sorted(f_b) == ["p", "rho", "u", "v", "w"]
    assert np.max(np.abs(pts_a - pts_b)) <= 1e-6 * np.max(np.abs(pts_b))
    for k in f_b:
        assert np.max(np.abs(f_a[k] - f_b[k])) <= 1e-6 * np.max(np.abs(f_b[k])), k
    x, y, z, (mach, alpha, re, t), q = cases.read_plot3d_binary(db / "output.xyz", db / "output.q")
    IM, JM, KM = c.shape
    gx, gy, gz = (np.asarray(a).reshape(KM, JM, IM) for a in (c.x, c.y, c.z))
    assert np.array_equal(x, gx) and np.array_equal(y, gy) and np.array_equal(z, gz)
    t_ck, Q = cases.read_checkpoint(db / "checkpoint.dat")
    assert t == t_ck and mach == c.params["Mach"]
    assert np.array_equal(q, np.moveaxis(Q[2:-2, 2:-2, 2:-2, :], -1, 0))


def test_bc_option(tmp_path):
    c = cases.case_vortex(20, 14, 10)
    d = c.write(tmp_path / "char", nsteps=5, checkpoint_freq=5)
    _run(d, "--bc", "characteristic")
    _, Q = cases.read_checkpoint(d / "checkpoint.dat")
    g, _ = pair(c, bc_mode=BC_CHARACTERISTIC)
    g.set_time(0.0)
    assert g.run(5) == 5
    assert max(per_var_rel_linf(Q.reshape(-1), g.get_conservative())) <= 1e-12
