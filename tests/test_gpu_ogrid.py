"""The O-grid boundary mode (BC_OGRID: i wraps around, wall on j = 0,
characteristic far field on j = JM-1) on a small NACA 0012 O-grid:

* the CUDA path matches the oracle's O-grid mode to the plain path's 1e-10
  after 20 steps, graph and per-call paths, inviscid and viscous (rho w,
  zero up to rounding in the inviscid runs, against the state's scale);
* the copied nodes either side of the seam equal the nodes they copy, bit for
  bit;
* moving the seam around the profile gives the same state, rolled;
* O-grid blocks are refused by a batch, and a block too short for the wrap
  by cbns_create.
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import OGRID_WRAP, Batch, Block, CbnsError, cases, make_params
from tests.helpers import per_var_rel_linf
from tests.test_gpu_parity import pair

pytestmark = pytest.mark.gpu
W = OGRID_WRAP


def _case(viscous, seam_shift=0):
    c = cases.case_naca_ogrid(48, 20, 4, first=2.0e-3, viscous=viscous)
    if seam_shift:
        c.x, c.y, c.z = (cases.ogrid_wrap(np.roll(a[..., W:-W], -seam_shift, axis=-1)) for a in (c.x, c.y, c.z))
    return c


def _run(g, n, graph):
    if graph:
        g.set_time(0.0)
        assert g.run(n) == n
    else:
        t = 0.0
        for _ in range(n):
            t = g.step_like_reference(t, 1.0e30)


@pytest.mark.parametrize("viscous", [False, True])
@pytest.mark.parametrize("graph", [False, True])
def test_ogrid_matches_oracle(viscous, graph):
    c = _case(viscous)
    g, o = pair(c)
    n = 20
    _run(g, n, graph)
    rc, _, no = o.solve(n, 1.0e30)
    assert rc == 0 and no == n
    q = g.get_conservative()
    ref = o.get_conservative()
    assert np.all(np.isfinite(q))
    # rho w of the extruded 2-D flow is zero up to rounding in inviscid runs
    # (~4e-17: the characteristic projection's round trip), so its difference is
    # held to 1e-10 of the state's scale, the other variables to 1e-10 of their own
    err = per_var_rel_linf(q, ref)
    assert max(err[:3] + err[4:]) <= 1e-10
    assert np.max(np.abs(q.reshape(-1, 5)[:, 3] - ref.reshape(-1, 5)[:, 3])) <= 1e-10 * np.max(np.abs(ref))
    IM, JM, KM = c.shape
    q = q.reshape(KM + 4, JM + 4, IM + 4, 5)
    P = IM - 2 * W
    for i in list(range(-2, W)) + list(range(IM - W, IM + 2)):
        src = i + P if i < W else i - P
        assert np.array_equal(q[:, :, i + 2], q[:, :, src + 2]), i


def test_seam_is_invisible():
    s = 13
    a, b = _case(True), _case(True, seam_shift=s)
    qs = []
    for c in (a, b):
        g, _ = pair(c)
        _run(g, 10, True)
        IM, JM, KM = c.shape
        qs.append(g.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)[:, :, 2 + W:IM + 2 - W])
    assert max(per_var_rel_linf(np.roll(qs[0], -s, axis=2).reshape(-1), qs[1].reshape(-1))) <= 1e-12


def test_ogrid_refusals():
    c = _case(True)
    g, _ = pair(c)
    with pytest.raises(CbnsError):
        Batch([g])
    with pytest.raises(CbnsError):
        Block(make_params(2 * W + 5, 12, 4, bc_mode=3))
