"""The oracle's far-field boundary mode (BC_FARFIELD): over steps, every
boundary and ghost node keeps the state it was set to, the interior evolves,
and with no vortex on a Cartesian box the free stream stays uniform to
round-off."""
import numpy as np

from cbns3d_cuda_b200 import BC_FARFIELD, CBNS_Q, cases, make_params
from oracle import oracle as orc


def _oracle(case, Q):
    o = orc.OracleBlock(make_params(*case.shape, **case.params, bc_mode=BC_FARFIELD))
    o.calc_metrics(case.x, case.y, case.z)
    o.set_conservative(Q)
    o.set_bc_calc_primitive(CBNS_Q)
    return o


def test_oracle_farfield_holds_the_boundary(oracle_lib):
    c = cases.case_vortex(24, 16, 10)
    IM, JM, KM = c.shape
    o = _oracle(c, c.Q0)
    q0 = o.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5).copy()
    rc, _, n = o.solve(5, 1.0e30)
    assert rc == 0 and n == 5
    q = o.get_conservative().reshape(q0.shape)
    shell = np.ones(q0.shape[:3], dtype=bool)
    shell[3:KM + 1, 3:JM + 1, 3:IM + 1] = False
    assert np.array_equal(q[shell], q0[shell])
    assert np.max(np.abs(q[~shell] - q0[~shell])) > 1e-6  # the vortex moves


def test_oracle_farfield_keeps_free_stream(oracle_lib):
    # on a Cartesian box (the metrics of the perturbed box do not preserve a
    # free stream, as the reference's do not)
    c = cases.case_vortex(20, 14, 10)
    c.x, c.y, c.z = cases.perturbed_box(20, 14, 10, amp=0.0)
    IM, JM, KM = c.shape
    g = c.params["gamma"]
    Q = np.zeros((KM + 4, JM + 4, IM + 4, 5))
    p_inf = 1.0 / (g * c.params["Mach"] ** 2)
    Q[..., 0] = 1.0
    Q[..., 1] = 1.0
    Q[..., 4] = p_inf / (g - 1.0) + 0.5
    o = _oracle(c, Q.reshape(-1))
    rc, _, n = o.solve(5, 1.0e30)
    assert rc == 0 and n == 5
    assert np.max(np.abs(o.get_conservative() - Q.reshape(-1))) <= 1e-8
