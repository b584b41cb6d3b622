"""Host-side logic: file formats, the .ini parser, case generators."""
import struct

import numpy as np
import pytest

from cbns3d_cuda_b200 import cases, make_params
from oracle import oracle as orc


def test_plot3d_roundtrip(tmp_path):
    x, y, z = cases.perturbed_box(7, 5, 6)
    cases.write_plot3d(tmp_path / "g.xyz", x, y, z)
    head = (tmp_path / "g.xyz").read_text().splitlines()[0]
    assert head.split() == ["7", "5", "6"]
    a, b, c = cases.read_plot3d(tmp_path / "g.xyz")
    assert np.array_equal(a, x) and np.array_equal(b, y) and np.array_equal(c, z)


def test_checkpoint_layout(tmp_path):
    Q = np.random.default_rng(0).random((8, 7, 6, 5))
    cases.write_checkpoint(tmp_path / "c.dat", 0.25, Q)
    raw = (tmp_path / "c.dat").read_bytes()
    t, IG, JG, KG = struct.unpack("<d3I", raw[:20])
    assert (t, IG, JG, KG) == (0.25, 6, 7, 8)
    assert len(raw) == 20 + 8 * Q.size
    # variable index fastest: n + 5*(i + IG*(j + JG*k))
    flat = np.frombuffer(raw[20:], dtype="<f8")
    assert flat[3 + 5 * (2 + IG * (1 + JG * 4))] == Q[4, 1, 2, 3]
    t2, Q2 = cases.read_checkpoint(tmp_path / "c.dat")
    assert t2 == 0.25 and np.array_equal(Q2, Q)


def test_input_txt_order(tmp_path):
    vals = dict(grid_fname="g.xyz", checkpoint_fname="c.dat", CFL=0.5, t_cur=0.0, t_end=1.0, Pr=0.72, Pr_t=0.9,
                gamma=1.4, Mach=0.5, Re=1e4, T_inf=288.15, angle_attack=1.25, nstep_max=10, checkpoint_freq=5,
                i_begin=1, i_end=0, is_restart=True)
    cases.write_input(tmp_path / "input.txt", **vals)
    lines = (tmp_path / "input.txt").read_text().split()
    assert lines[0] == "g.xyz" and lines[11] == "1.25" and lines[16] == "1" and len(lines) == 17
    with pytest.raises(ValueError):
        cases.write_input(tmp_path / "x.txt", CFL=0.5)


def test_parse_ini_matches_reference_parser(tmp_path):
    """python/parser_ini.py writes each value in section order, one per line."""
    ini = tmp_path / "case.ini"
    ini.write_text("[string]\ngrid_fname = grid.xyz\ncheckpoint_fname = checkpoint.dat\n\n[real]\nCFL = 0.8\n"
                   "t_cur = 0.0\nt_end = 100.0\n\n[integer]\nnstep_max = 10\n\n[bool]\nis_restart = 1\n")
    cases.parse_ini(ini, tmp_path / "input.txt")
    assert (tmp_path / "input.txt").read_text().split("\n")[:-1] == [
        "grid.xyz", "checkpoint.dat", "0.8", "0.0", "100.0", "10", "1"]


@pytest.mark.parametrize("make", [lambda: cases.case_vortex(20, 14, 10), lambda: cases.case_naca(40, 20, 6),
                                  lambda: cases.case_blast(16, 16, 16), lambda: cases.case_shock_vortex(24, 20, 8)])
def test_case_grids_right_handed_and_states_physical(oracle_lib, make):
    c = make()
    IM, JM, KM = c.shape
    o = orc.OracleBlock(make_params(IM, JM, KM))
    o.calc_metrics(c.x, c.y, c.z)
    J = o.get_metrics()[9]
    assert (J > 0).all()
    if c.Q0 is not None:
        r, u, v, w, p = cases.primitive(c.Q0, 1.4)
        assert (r > 0).all() and (p > 0).all() and np.isfinite(c.Q0).all()


def test_naca_grid_spacing():
    x, y, z, r = cases.naca0012_ogrid(64, 32, 4)
    # first wall-normal spacing 1e-5 chords and outer radius ~20 chords
    d1 = np.hypot(x[0, 1] - x[0, 0], y[0, 1] - y[0, 0])
    assert np.allclose(d1, 1e-5, rtol=1e-6)
    dist = np.hypot(x[0, -1] - x[0, 0], y[0, -1] - y[0, 0])
    assert np.allclose(dist, 20.0)
    assert 1.0 < r < 2.0


def test_naca_blend_grid_and_wrap(oracle_lib):
    """The O-grid of the wrap-around mode: right-handed with its wrap copies
    (metrics of the O-grid mode), wall spacing `first` of each line's length,
    outer points on the 20-chord circle, and the seam cells no larger than
    their neighbours around the profile."""
    P, JM, KM = 64, 32, 4
    x, y, z = cases.naca0012_ogrid_blend(P, JM, KM, first=1e-5)
    L = np.hypot(x[0, -1] - x[0, 0], y[0, -1] - y[0, 0])
    d1 = np.hypot(x[0, 1] - x[0, 0], y[0, 1] - y[0, 0])
    assert np.allclose(d1, 1e-5 * L / 20.0, rtol=1e-6)  # first / far of the line's length L
    assert np.allclose(np.hypot(x[0, -1] - 0.5, y[0, -1]), 20.0)
    ds = np.hypot(np.diff(x[0, 8], append=x[0, 8, :1]), np.diff(y[0, 8], append=y[0, 8, :1]))
    assert ds[-1] <= 1.5 * max(ds[-2], ds[0])  # the cell across the trailing edge
    c = cases.case_naca_ogrid(P, JM, KM)
    assert c.shape == (P + 8, JM, KM)
    assert np.array_equal(c.x[..., :4], x[..., -4:]) and np.array_equal(c.x[..., -4:], x[..., :4])
    o = orc.OracleBlock(make_params(*c.shape, **c.params))
    o.calc_metrics(c.x, c.y, c.z)
    J = o.get_metrics()[9]
    assert (J > 0).all()


def _write_vtk(path, dims, pts, fields, binary):
    """The driver's legacy VTK layout (Block3d::output_vtk / output_vtk_binary)."""
    n = pts.shape[0]
    with open(path, "wb") as f:
        f.write(b"# vtk DataFile Version 3.0\nvtk output\n" + (b"BINARY" if binary else b"ASCII") +
                b"\nDATASET STRUCTURED_GRID\n")
        f.write(f"DIMENSIONS {dims[0]} {dims[1]} {dims[2]}\nPOINTS {n} double\n".encode())
        if binary:
            f.write(pts.astype(">f8").tobytes() + b"\n")
        else:
            f.write("".join(f"{a:E} {b:E} {c:E}\n" for a, b, c in pts).encode())
        f.write(f"POINT_DATA {n}\nFIELD FieldData {len(fields)}\n".encode())
        for name, v in fields.items():
            f.write(f"{name} 1 {n} double\n".encode())
            if binary:
                f.write(v.astype(">f8").tobytes() + b"\n")
            else:
                f.write("".join(f"{a:E}\n" for a in v).encode())


def test_read_vtk_ascii_and_binary(tmp_path):
    rng = np.random.default_rng(0)
    dims = (4, 3, 2)
    n = 24
    pts = rng.standard_normal((n, 3))
    fields = {k: rng.standard_normal(n) for k in ("rho", "u", "v", "w", "p")}
    for binary in (False, True):
        path = tmp_path / f"o{int(binary)}.vtk"
        _write_vtk(path, dims, pts, fields, binary)
        d, p, f = cases.read_vtk(path)
        assert d == dims and sorted(f) == sorted(fields)
        # BINARY is exact; ASCII carries %E's 7 significant digits
        tol = 0.0 if binary else 1e-6
        assert np.max(np.abs(p - pts)) <= tol * np.max(np.abs(pts))
        for k in fields:
            assert np.max(np.abs(f[k] - fields[k])) <= tol * np.max(np.abs(fields[k]))


def test_naca_marched_grid_full_size(oracle_lib):
    """The marched O-grid at the NACA configuration's size: positive Jacobian
    everywhere (O-grid metrics), first cell 1e-5, lines leaving the wall within
    a few degrees of its normal, outer boundary about 20 chords out."""
    c = cases.case_naca_ogrid(384, 128, 4, grid="marched")
    x, y = c.x[0, :, 4:-4], c.y[0, :, 4:-4]
    d1 = np.hypot(x[1] - x[0], y[1] - y[0])
    assert np.allclose(d1, 1e-5, rtol=1e-9)
    tx, ty = np.roll(x[0], -1) - np.roll(x[0], 1), np.roll(y[0], -1) - np.roll(y[0], 1)
    cosang = ((x[1] - x[0]) * tx + (y[1] - y[0]) * ty) / (d1 * np.hypot(tx, ty))
    assert np.max(np.abs(cosang)) < 0.1  # within ~6 degrees of the wall normal
    r = np.hypot(x[-1] - 0.5, y[-1])
    assert 19.0 < r.min() and r.max() < 21.0
    o = orc.OracleBlock(make_params(*c.shape, **c.params))
    o.calc_metrics(c.x, c.y, c.z)
    assert (np.asarray(o.get_metrics()[9]) > 0).all()
