"""The oracle's hybrid flux (face mask + linear upwind-5 flux) on known answers.

* a mask of all ones is the WENO5 flux, bit for bit;
* in uniform flow and on a linear density ramp both reconstructions are exact,
  so the linear flux equals WENO5 to round-off;
* at a shock the linear flux differs from WENO5 (the mask is in effect), and
  a masked face changes only the two nodes that share it.
"""
import numpy as np

from cbns3d_cuda_b200 import CBNS_Q, cases, make_params
from oracle import oracle as orc


def _oracle(case, Q=None):
    o = orc.OracleBlock(make_params(*case.shape, **case.params))
    o.calc_metrics(case.x, case.y, case.z)
    o.set_conservative(case.Q0 if Q is None else Q)
    o.set_bc_calc_primitive(CBNS_Q)
    return o


def _nfaces(IM, JM, KM):
    return (IM - 1) * (JM - 2) * (KM - 2) + (IM - 2) * (JM - 1) * (KM - 2) + (IM - 2) * (JM - 2) * (KM - 1)


def test_all_ones_mask_is_weno(oracle_lib):
    c = cases.case_blast(16, 16, 16)
    o = _oracle(c)
    ref = o.eval_rhs(CBNS_Q)
    o.set_face_mask(np.ones(_nfaces(*c.shape), np.uint8))
    assert np.array_equal(o.eval_rhs(CBNS_Q), ref)


def test_linear_equals_weno_on_uniform_and_ramp(oracle_lib):
    c = cases.case_vortex(14, 12, 8)
    IM, JM, KM = c.shape
    Q = np.asarray(c.Q0).reshape(KM + 4, JM + 4, IM + 4, 5).copy()
    # uniform flow (u 0.5, p = p_inf, the value the i-face boundary resets
    # to) with a density ramp along i; compared away from the boundaries
    g = 1.4
    p_inf = 1.0 / (g * c.params["Mach"] ** 2)
    ramp = 1.0 + 0.01 * np.arange(IM + 4)[None, None, :]
    rho = np.broadcast_to(ramp, Q.shape[:3])
    Q[..., 0] = rho
    Q[..., 1] = 0.5 * rho
    Q[..., 2] = 0.0
    Q[..., 3] = 0.0
    Q[..., 4] = p_inf / (g - 1) + 0.5 * rho * 0.25
    o = _oracle(c, Q.reshape(-1))
    ref = o.eval_rhs(CBNS_Q).reshape(KM - 2, JM - 2, IM - 2, 5)
    o.set_face_mask(np.zeros(_nfaces(*c.shape), np.uint8))
    lin = o.eval_rhs(CBNS_Q).reshape(KM - 2, JM - 2, IM - 2, 5)
    # the i-face boundary rewrites the boundary nodes too: stay 3 nodes clear
    w = (slice(2, -2), slice(2, -2), slice(3, -3))
    assert np.max(np.abs(ref[w])) > 1e-6  # the ramp is advected: a non-zero right-hand side
    assert np.max(np.abs(lin[w] - ref[w])) <= 1e-9 * np.max(np.abs(ref[w]))


def test_linear_differs_at_shock_and_locally(oracle_lib):
    c = cases.case_shock_vortex(40, 36, 12)
    IM, JM, KM = c.shape
    o = _oracle(c)
    ref = o.eval_rhs(CBNS_Q).reshape(KM - 2, JM - 2, IM - 2, 5)
    o.set_face_mask(np.zeros(_nfaces(*c.shape), np.uint8))
    lin = o.eval_rhs(CBNS_Q).reshape(KM - 2, JM - 2, IM - 2, 5)
    d = np.abs(lin - ref).max(axis=(0, 1, 3))  # per i column
    assert d.max() > 1e-3 * np.abs(ref).max()
    # one linear i-face (low node i = 20 of row j = 6, k = 5, at the shock)
    # changes exactly the two nodes that share it
    i, j, k = 20, 6, 5
    m = np.ones(_nfaces(*c.shape), np.uint8)
    m[i + (IM - 1) * ((j - 1) + (JM - 2) * (k - 1))] = 0
    o.set_face_mask(m)
    one = o.eval_rhs(CBNS_Q).reshape(KM - 2, JM - 2, IM - 2, 5)
    changed = np.argwhere(np.abs(one - ref).max(axis=-1) > 0)
    assert sorted(map(tuple, changed)) == [(k - 1, j - 1, i - 1), (k - 1, j - 1, i)]
