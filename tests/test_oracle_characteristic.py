"""The oracle's characteristic far-field mode (BC_CHARACTERISTIC), checked
through properties of the Riemann-invariant state it sets on the i faces of a
Cartesian box (outward normals -x and +x):

* subsonic outflow face: the outgoing invariant qn + 2c/(g-1) and the entropy
  p/rho^g equal the inward neighbour's, the incoming qn - 2c/(g-1) the free
  stream's, the tangential velocity is the neighbour's;
* subsonic inflow face: outgoing invariant from the neighbour, incoming one,
  entropy and tangential velocity from the free stream;
* supersonic: the inflow face takes the free stream, the outflow face copies
  the neighbour bit for bit; ghosts copy their boundary node;
* a uniform free stream stays uniform over steps;
* the boundary nodes depend on the buffer's interior only;
* an acoustic pulse leaves with less left behind than with held boundaries.
"""
import numpy as np

from cbns3d_cuda_b200 import BC_CHARACTERISTIC, CBNS_Q, cases, make_params
from oracle import oracle as orc


def _box(IM=20, JM=14, KM=10, Mach=0.5):
    c = cases.case_vortex(IM, JM, KM, Mach=Mach)
    c.x, c.y, c.z = cases.perturbed_box(IM, JM, KM, amp=0.0)
    return c


def _apply(c, Q):
    o = orc.OracleBlock(make_params(*c.shape, **c.params, bc_mode=BC_CHARACTERISTIC))
    o.calc_metrics(c.x, c.y, c.z)
    o.set_conservative(Q.reshape(-1))
    o.set_bc_calc_primitive(CBNS_Q)
    return o


def _prims(q, g):
    r = q[..., 0]
    u, v, w = q[..., 1] / r, q[..., 2] / r, q[..., 3] / r
    p = (g - 1.0) * (q[..., 4] - 0.5 * r * (u * u + v * v + w * w))
    return r, u, v, w, p


def test_subsonic_faces_follow_the_invariants(oracle_lib):
    c = _box()
    IM, JM, KM = c.shape
    g = c.params["gamma"]
    g1 = g - 1.0
    p_inf = 1.0 / (g * c.params["Mach"] ** 2)
    c_inf = np.sqrt(g * p_inf)
    q = _apply(c, c.Q0).get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)
    inner = (slice(3, KM + 1), slice(3, JM + 1))  # j, k away from the other faces
    for ib, ie, sgn in ((2, 3, -1.0), (IM + 1, IM, 1.0)):
        rb, ub, vb, wb, pb = _prims(q[inner + (ib,)], g)
        re, ue, ve, we, pe = _prims(q[inner + (ie,)], g)
        cb, ce = np.sqrt(g * pb / rb), np.sqrt(g * pe / re)
        qnb, qne, qni = sgn * ub, sgn * ue, sgn * 1.0
        assert np.all(np.abs(qne) < ce)
        np.testing.assert_allclose(qnb + 2 * cb / g1, qne + 2 * ce / g1, rtol=0, atol=1e-12)
        np.testing.assert_allclose(qnb - 2 * cb / g1, qni - 2 * c_inf / g1, rtol=0, atol=1e-12)
        if sgn > 0:  # outflow: entropy and tangential velocity of the neighbour
            assert np.all(qnb >= 0)
            np.testing.assert_allclose(pb / rb ** g, pe / re ** g, rtol=1e-12)
            np.testing.assert_allclose(vb, ve, rtol=0, atol=1e-13)
            np.testing.assert_allclose(wb, we, rtol=0, atol=1e-13)
        else:  # inflow: entropy and tangential velocity of the free stream
            assert np.all(qnb < 0)
            np.testing.assert_allclose(pb / rb ** g, p_inf, rtol=1e-12)
            np.testing.assert_allclose(vb, 0.0, rtol=0, atol=1e-13)
            np.testing.assert_allclose(wb, 0.0, rtol=0, atol=1e-13)
        for l in (1, 2):  # ghosts copy the boundary node
            gi = ib - l if sgn < 0 else ib + l
            assert np.array_equal(q[inner + (gi,)], q[inner + (ib,)])


def test_supersonic_faces(oracle_lib):
    c = _box(Mach=2.0)
    IM, JM, KM = c.shape
    g = c.params["gamma"]
    p_inf = 1.0 / (g * 4.0)
    Q = np.zeros((KM + 4, JM + 4, IM + 4, 5))
    rng = np.random.default_rng(3)
    Q[..., 0] = 1.0 + 0.05 * rng.random(Q.shape[:3])
    Q[..., 1] = Q[..., 0] * 1.0
    Q[..., 4] = p_inf / (g - 1.0) + 0.5 * Q[..., 0]
    q = _apply(c, Q).get_conservative().reshape(Q.shape)
    inner = (slice(3, KM + 1), slice(3, JM + 1))
    free = np.array([1.0, 1.0, 0.0, 0.0, p_inf / (g - 1.0) + 0.5])
    for i in (0, 1, 2):  # inflow face and its ghosts
        np.testing.assert_allclose(q[inner + (i,)], np.broadcast_to(free, q[inner + (i,)].shape), rtol=1e-15, atol=1e-15)
    for i in (IM + 1, IM + 2, IM + 3):  # outflow face and ghosts copy i = IM-2
        assert np.array_equal(q[inner + (i,)], Q[inner + (IM,)])


def test_free_stream_stays_uniform(oracle_lib):
    c = _box()
    IM, JM, KM = c.shape
    g = c.params["gamma"]
    p_inf = 1.0 / (g * c.params["Mach"] ** 2)
    Q = np.zeros((KM + 4, JM + 4, IM + 4, 5))
    Q[..., 0] = 1.0
    Q[..., 1] = 1.0
    Q[..., 4] = p_inf / (g - 1.0) + 0.5
    o = _apply(c, Q)
    rc, _, n = o.solve(5, 1.0e30)
    assert rc == 0 and n == 5
    assert np.max(np.abs(o.get_conservative() - Q.reshape(-1))) <= 1e-8


def test_state_depends_on_the_interior_only(oracle_lib):
    # two buffers with the same interior and different boundary and ghost
    # values give the same boundary nodes: the phases read only nodes that are
    # interior or set earlier in the same call (the graph path rotates three
    # buffers with different histories)
    c = _box(Mach=0.5)
    c.x, c.y, c.z = cases.perturbed_box(*c.shape)
    IM, JM, KM = c.shape
    Q1 = c.Q0.reshape(KM + 4, JM + 4, IM + 4, 5).copy()
    Q2 = Q1.copy()
    shell = np.ones(Q1.shape[:3], dtype=bool)
    shell[3:KM + 1, 3:JM + 1, 3:IM + 1] = False
    rng = np.random.default_rng(5)
    Q2[shell] *= 1.0 + 0.05 * rng.random((int(shell.sum()), 1))
    a = _apply(c, Q1).get_conservative().reshape(Q1.shape)
    b = _apply(c, Q2).get_conservative().reshape(Q1.shape)
    face = np.zeros_like(shell)
    face[2:KM + 2, 2:JM + 2, 2:IM + 2] = True
    face &= shell
    assert np.array_equal(a[face], b[face])
    assert np.array_equal(a[~shell], b[~shell])


def test_pulse_leaves_with_less_left_behind_than_the_held_far_field(oracle_lib):
    # a spherical acoustic pulse (1e-3 of p_inf) in a Mach 0.5 stream through a
    # 4^3 box: at t = 5, when it has crossed every face, 1.6e-3 of it remains
    # with the characteristic far field, 2.3e-3 with boundaries that hold the
    # free stream
    from cbns3d_cuda_b200 import BC_FARFIELD
    N = 21
    c = cases.case_vortex(N, N, N, Mach=0.5)
    c.x, c.y, c.z = cases.perturbed_box(N, N, N, L=(4.0, 4.0, 4.0), amp=0.0)
    g = c.params["gamma"]
    p_inf = 1.0 / (g * 0.25)
    eps = 1e-3
    pp = p_inf * (1 + eps * np.exp(-((c.x - 2.0) ** 2 + (c.y - 2.0) ** 2 + (c.z - 2.0) ** 2) / 0.16))
    rho = (pp / p_inf) ** (1 / g)
    Q = np.zeros((N + 4, N + 4, N + 4, 5))
    Q[..., 0] = 1.0
    Q[..., 1] = 1.0
    Q[..., 4] = p_inf / (g - 1) + 0.5
    grid = (slice(2, N + 2),) * 3
    Q[grid + (0,)] = rho
    Q[grid + (1,)] = rho
    Q[grid + (4,)] = pp / (g - 1) + 0.5 * rho
    left = {}
    for mode in (BC_FARFIELD, BC_CHARACTERISTIC):
        o = orc.OracleBlock(make_params(N, N, N, **c.params, bc_mode=mode))
        o.calc_metrics(c.x, c.y, c.z)
        o.set_conservative(Q.reshape(-1))
        o.set_bc_calc_primitive(CBNS_Q)
        rc, _, n = o.solve(100000, 5.0)
        assert rc == 0 and n > 300
        r, u, v, w, p = _prims(o.get_conservative().reshape(Q.shape)[grid], g)
        left[mode] = np.max(np.abs(p / p_inf - 1.0)) / eps
    assert left[BC_CHARACTERISTIC] < 0.8 * left[BC_FARFIELD]
    assert left[BC_CHARACTERISTIC] < 5e-3
