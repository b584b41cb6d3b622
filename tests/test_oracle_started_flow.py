"""The NACA 0012 configuration's started flow and full viscous time-step limit,
on the CPU:

* the panel method's potential flow has zero normal velocity at the panel
  midpoints, meets the Kutta condition at the trailing edge, recovers the
  free stream far away and gives the known incompressible NACA 0012 answers
  (suction peak Cp ~ -0.41 near x/c 0.12 at zero incidence; lift slope of a
  12% section, Cl ~ 0.150 at 1.25 deg);
* the started state is positive, at rest on the wall, tangent to the wall on
  the first node lines and the free stream at the far boundary;
* the oracle's dt with dt_viscous = FULL is at most the reference formula's,
  and the same in an inviscid run.
"""
import numpy as np

from cbns3d_cuda_b200 import CBNS_Q, DTV_FULL, DTV_REFERENCE, cases, make_params
from oracle import oracle as orc


def _panels(n=256):
    xs, ys = cases.naca0012_rounded_surface(n)
    x1, y1 = np.roll(xs, -1), np.roll(ys, -1)
    th = np.arctan2(y1 - ys, x1 - xs)
    return xs, ys, x1, y1, th


def _surface_velocity(alpha, n=256, off=1e-6):
    xs, ys, x1, y1, th = _panels(n)
    vel = cases.panel_flow(xs, ys, alpha)
    xm, ym = 0.5 * (xs + x1) - off * np.sin(th), 0.5 * (ys + y1) + off * np.cos(th)
    u, v = vel(xm, ym)
    return xs, ys, x1, y1, th, xm, u, v


def test_panel_flow_normal_velocity_and_kutta():
    # just outside the panel midpoints (the self-influence branch of the solver
    # applies on the surface itself)
    xs, ys, x1, y1, th, xm, u, v = _surface_velocity(1.25, off=1e-9)
    vn = -u * np.sin(th) + v * np.cos(th)
    vt = u * np.cos(th) + v * np.sin(th)
    assert np.max(np.abs(vn)) < 1e-6
    assert abs(vt[0] + vt[-1]) < 1e-6 * max(1.0, abs(vt[0]))
    # the flow leaves the trailing edge: towards it on both panels
    assert vt[0] < 0 < vt[-1]


def test_panel_flow_known_answers():
    xs, ys, x1, y1, th, xm, u, v = _surface_velocity(0.0, n=384, off=1e-4)
    cp = 1.0 - (u * u + v * v)
    assert -0.43 < cp.min() < -0.40
    assert 0.08 < xm[np.argmin(cp)] < 0.16
    xs, ys, x1, y1, th, xm, u, v = _surface_velocity(1.25, n=384, off=1e-4)
    cp = 1.0 - (u * u + v * v)
    L = np.hypot(x1 - xs, y1 - ys)
    fx, fy = (-cp * -np.sin(th) * L).sum(), (-cp * np.cos(th) * L).sum()
    al = np.deg2rad(1.25)
    cl = fy * np.cos(al) - fx * np.sin(al)
    assert 0.14 < cl < 0.16
    vel = cases.panel_flow(*cases.naca0012_rounded_surface(384), 1.25)
    uf, vf = vel(np.array([200.0]), np.array([-50.0]))
    assert abs(uf[0] - np.cos(al)) < 1e-3 and abs(vf[0] - np.sin(al)) < 1e-3


def test_started_state():
    c = cases.case_naca_ogrid(96, 40, 4, grid="marched", first=1e-4, start="potential")
    assert c.params["vis_divergence"] == 1 and c.params["dt_viscous"] == 1
    Q = c.Q0
    IM, JM, KM = c.shape
    assert Q.shape == (KM + 4, JM + 4, IM + 4, 5)
    q = Q[2:-2, 2:-2, 2:-2]
    r = q[..., 0]
    u, v = q[..., 1] / r, q[..., 2] / r
    p = 0.4 * (q[..., 4] - 0.5 * r * (u * u + v * v))
    assert np.all(r > 0) and np.all(p > 0)
    assert np.all(u[:, 0] == 0) and np.all(v[:, 0] == 0)
    # tangent to the wall on the first line of nodes
    X, Y = c.x[0], c.y[0]
    tx, ty = np.roll(X[0], -1) - np.roll(X[0], 1), np.roll(Y[0], -1) - np.roll(Y[0], 1)
    n = np.hypot(tx, ty)
    vn = (-u[0, 1] * ty + v[0, 1] * tx) / n
    assert np.max(np.abs(vn)) < 0.05
    # far boundary: the free stream within a few percent, p_inf = 1/(gamma M^2)
    al = np.deg2rad(1.25)
    assert np.max(np.abs(u[:, -1] - np.cos(al))) < 0.02
    assert np.max(np.abs(p[:, -1] * 1.4 * 0.64 - 1.0)) < 0.03


def _dt(viscous, dtv):
    c = cases.case_naca_ogrid(48, 20, 4, first=2.0e-3, viscous=viscous)
    o = orc.OracleBlock(make_params(*c.shape, **c.params, dt_viscous=dtv))
    o.init_like_reference(c.x, c.y, c.z)
    # advance a few steps so the wall has slowed the flow next to it
    rc, _, _ = o.solve(3, 1.0e30)
    assert rc == 0
    dt = o.calc_dt()
    o.close()
    return dt


def test_full_viscous_dt_limit():
    d_ref, d_full = _dt(True, DTV_REFERENCE), _dt(True, DTV_FULL)
    assert 0 < d_full < d_ref
    assert _dt(False, DTV_REFERENCE) == _dt(False, DTV_FULL)
