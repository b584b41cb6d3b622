"""End-to-end parity with the reference build on the same B200.

The unmodified reference executables (oracle/_ref, compiled from the
reference sources by `make -C oracle ref`) and this project's driver
(cbns3d_cuda_b200/bin/cbns3d_b200, which calls the CUDA library through the
block3d_cuda shims) read the same input.txt, Plot3D grid and checkpoint; the
checkpoints they write must agree to relative L-infinity <= 1e-10 per
variable after 100 steps (isentropic vortex, inviscid), 20 steps (the
shock-vortex case of the throughput benchmark at 128 x 128 x 64, inviscid) and
50 steps (NACA, viscous), and the VTK files must have the same layout with
values equal to their printed precision.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cbns3d_cuda_b200 import cases
from tests.helpers import per_var_rel_linf

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref"
EXE = ROOT / "cbns3d_cuda_b200" / "bin" / "cbns3d_b200"


def run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def vtk_fields(path):
    lines = Path(path).read_text().splitlines()
    head = lines[:6]
    out = {}
    i = 0
    while i < len(lines):
        parts = lines[i].split()
        if len(parts) == 4 and parts[1] == "1" and parts[3] == "double":
            n = int(parts[2])
            out[parts[0]] = np.array([float(v) for v in lines[i + 1:i + 1 + n]])
            i += n
        i += 1
    return head, out


CASES = {
    "vortex_c0": (lambda: cases.case_vortex(64, 32, 16), 100, "inv"),
    "naca_viscous": (lambda: cases.case_naca(64, 32, 6, first=1e-3), 50, "visc"),
    "shock_vortex_mid": (lambda: cases.case_shock_vortex(128, 128, 64), 20, "inv"),
}
# the programs compared with the reference build on identical inputs
VARIANTS = {
    "driver": lambda mode: [str(EXE), "--quiet", "--inviscid" if mode == "inv" else "--viscous"],
    "driver_graph": lambda mode: [str(EXE), "--quiet", "--graph", "--inviscid" if mode == "inv" else "--viscous"],
    # the reference's own src/Block3d.cpp + src/cbns3d.cpp, unmodified, linked to libcbns_b200
    "reference_host_dropin": lambda mode: [str(REF / f"cbns3d_dropin_{mode}")],
}
_ref_cache = {}


def reference_output(name, tmp_root):
    if name not in _ref_cache:
        make, n, mode = CASES[name]
        c = make()
        d = c.write(tmp_root / f"ref_{name}", nsteps=n, checkpoint_freq=n)
        out = run([str(REF / f"cbns3d_ref_{mode}")], d)
        assert "Elapsed Time" in out
        _ref_cache[name] = (c, d)
    return _ref_cache[name]


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_matches_reference_build(tmp_path_factory, name, variant):
    make, n, mode = CASES[name]
    if not (REF / f"cbns3d_ref_{mode}").exists():
        pytest.skip("reference build absent (make -C oracle ref needs the reference sources)")
    cmd = VARIANTS[variant](mode)
    if not Path(cmd[0]).exists():
        pytest.skip(f"{cmd[0]} not built")
    c, dref = reference_output(name, tmp_path_factory.getbasetemp())
    dmine = c.write(tmp_path_factory.mktemp(variant), nsteps=n, checkpoint_freq=n)
    out_mine = run(cmd, dmine)
    assert "Elapsed Time" in out_mine
    t_r, Q_r = cases.read_checkpoint(dref / "checkpoint.dat")
    t_m, Q_m = cases.read_checkpoint(dmine / "checkpoint.dat")
    assert abs(t_r - t_m) <= 1e-12 * abs(t_r)
    err = per_var_rel_linf(Q_m, Q_r)
    assert max(err) <= 1e-10, err
    h_r, f_r = vtk_fields(dref / "output.vtk")
    h_m, f_m = vtk_fields(dmine / "output.vtk")
    assert h_r == h_m
    assert sorted(f_r) == sorted(f_m) == ["p", "rho", "u", "v", "w"]
    for k in f_r:
        assert np.allclose(f_m[k], f_r[k], rtol=2e-6, atol=1e-12), k
