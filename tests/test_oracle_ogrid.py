"""The oracle's O-grid boundary mode (BC_OGRID) on a small NACA 0012 O-grid:

* after a boundary pass every copied node (i < 4, i >= IM-4, i ghosts) equals
  the node P away, bit for bit;
* the seam is invisible: moving the seam by s points around the profile
  (the same grid, its periodic line rolled) gives, after some steps, the same
  state rolled by s, bit for bit, inviscid and viscous;
* the wall holds: zero velocity on j = 0 in viscous runs.

The grid is naca0012_ogrid_blend: on the surface-normal O-grid the single
cell across a sharp trailing edge turns by almost 180 degrees, and a run
wrapped across it loses positivity within ten steps.
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import BC_OGRID, CBNS_Q, OGRID_WRAP, cases, make_params
from oracle import oracle as orc

W = OGRID_WRAP


def _case(viscous, seam_shift=0, P=48, JM=20, KM=4):
    c = cases.case_naca_ogrid(P, JM, KM, first=2.0e-3, viscous=viscous)
    if seam_shift:
        c.x, c.y, c.z = (cases.ogrid_wrap(np.roll(a[..., W:-W], -seam_shift, axis=-1)) for a in (c.x, c.y, c.z))
    return c


def _oracle(c):
    o = orc.OracleBlock(make_params(*c.shape, **c.params))
    o.calc_metrics(c.x, c.y, c.z)
    o.initial_condition()
    o.calc_conservative(CBNS_Q)
    if c.params["viscous"]:
        o.calc_primitive(CBNS_Q)
    o.set_bc_calc_primitive(CBNS_Q)
    return o


def _q(o, c):
    IM, JM, KM = c.shape
    return o.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)


def test_copies_across_the_seam(oracle_lib):
    c = _case(True)
    o = _oracle(c)
    rc, _, n = o.solve(3, 1.0e30)
    assert rc == 0 and n == 3
    q = _q(o, c)
    IM = c.shape[0]
    P = IM - 2 * W
    for i in list(range(-2, W)) + list(range(IM - W, IM + 2)):
        src = i + P if i < W else i - P
        assert np.array_equal(q[:, :, i + 2], q[:, :, src + 2]), i


@pytest.mark.parametrize("viscous", [False, True])
def test_seam_is_invisible(oracle_lib, viscous):
    s = 13
    a, b = _case(viscous), _case(viscous, seam_shift=s)
    oa, ob = _oracle(a), _oracle(b)
    for o in (oa, ob):
        rc, _, n = o.solve(20, 1.0e30)
        assert rc == 0 and n == 20
    qa, qb = _q(oa, a), _q(ob, b)
    assert np.all(np.isfinite(qa)) and np.all(np.isfinite(qb))
    IM = a.shape[0]
    ca = qa[:, :, 2 + W:IM + 2 - W]
    cb = qb[:, :, 2 + W:IM + 2 - W]
    assert np.all(np.isfinite(ca))
    assert np.array_equal(np.roll(ca, -s, axis=2), cb)


def test_wall_holds(oracle_lib):
    c = _case(True)
    o = _oracle(c)
    rc, _, n = o.solve(4, 1.0e30)
    assert rc == 0 and n == 4
    q = _q(o, c)
    assert np.all(q[2:-2, 2, 2:-2, 1:4] == 0.0)
    assert np.max(np.abs(q[2:-2, 3, 2:-2, 1:4])) > 0.0
