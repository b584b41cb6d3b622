"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 comparisons use the relative L-infinity norm (max |a-b| / max |b|) per
conservative variable: single operations <= 1e-12, 20-100 RK3 steps <= 1e-10
(the bound the plain path must meet against the reference build).  The split
precision path is held to a density L2 error <= 1e-5 relative to the FP64
oracle run.
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, CBNS_QP, PREC_SPLIT, VISDIV_CENTERED, Block, cases, make_params
from cbns3d_cuda_b200._abi import CBNS_ERR_NAN_DT, CbnsError
from oracle import oracle as orc
from tests.helpers import interior, per_var_rel_linf, rel_linf

pytestmark = pytest.mark.gpu


def pair(case, **over):
    p = dict(case.params)
    p.update(over)
    IM, JM, KM = case.shape
    prm = make_params(IM, JM, KM, **p)
    g = Block(prm)
    o = orc.OracleBlock(make_params(IM, JM, KM, **{k: v for k, v in p.items() if k != "precision"}))
    for b in (g, o):
        b.calc_metrics(case.x, case.y, case.z)
        if case.Q0 is None:
            b.initial_condition()
            b.calc_conservative(CBNS_Q)
        else:
            b.set_conservative(case.Q0)
            if p.get("viscous"):
                b.calc_primitive(CBNS_Q)
        b.set_bc_calc_primitive(CBNS_Q)
        if p.get("viscous"):
            b.calc_viscous_terms()
    return g, o


# odd sizes exercise partial tiles in every direction
SHAPES = [(20, 14, 10), (37, 23, 9), (16, 31, 12)]


@pytest.mark.parametrize("shape", SHAPES)
def test_metrics(shape):
    c = cases.case_vortex(*shape)
    g, o = pair(c)
    assert rel_linf(g.get_metrics(), o.get_metrics()) <= 1e-13


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("wall", [False, True])
def test_boundary_conditions(shape, wall):
    c = cases.case_vortex(*shape)
    over = dict(i_end=shape[0]) if wall else {}
    g, o = pair(c, **over)
    for which in (CBNS_Q, CBNS_QP):
        assert rel_linf(g.get_conservative(which), o.get_conservative(which)) <= 1e-15


@pytest.mark.parametrize("shape", SHAPES)
def test_rhs_inviscid(shape):
    c = cases.case_vortex(*shape)
    g, o = pair(c)
    err = per_var_rel_linf(g.eval_rhs(CBNS_Q), o.eval_rhs(CBNS_Q))
    assert max(err) <= 1e-12, err


@pytest.mark.parametrize("visdiv", [0, VISDIV_CENTERED])
def test_rhs_viscous(visdiv):
    c = cases.case_vortex(21, 15, 10)
    g, o = pair(c, viscous=True, Re=300.0, i_end=21, vis_divergence=visdiv)
    err = per_var_rel_linf(g.eval_rhs(CBNS_Q), o.eval_rhs(CBNS_Q))
    assert max(err) <= 1e-12, err


def test_dt():
    c = cases.case_vortex(20, 14, 10)
    g, o = pair(c)
    assert abs(g.calc_dt() - o.calc_dt()) <= 1e-14 * o.calc_dt()
    gv, ov = pair(c, viscous=True, Re=100.0)
    assert abs(gv.calc_dt() - ov.calc_dt()) <= 1e-13 * ov.calc_dt()


def _steps(g, o, n, t_end=1e30, graph=False):
    t = 0.0
    if graph:
        g.set_time(0.0)
        assert g.run(n, t_end) == n
    else:
        for _ in range(n):
            t = g.step_like_reference(t, t_end)
    rc, to, no = o.solve(n, t_end)
    assert rc == 0 and no == n
    return to


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("shape,n", [((20, 14, 10), 20), ((64, 32, 16), 100)])
def test_steps_inviscid(shape, n, graph):
    c = cases.case_vortex(*shape)
    g, o = pair(c)
    to = _steps(g, o, n, graph=graph)
    if graph:
        t, _ = g.get_time()
        assert abs(t - to) <= 1e-12 * to
    for which in (CBNS_Q, CBNS_QP):
        err = per_var_rel_linf(g.get_conservative(which), o.get_conservative(which))
        assert max(err) <= 1e-10, (which, err)


@pytest.mark.parametrize("graph", [False, True])
def test_steps_wall_and_viscous(graph):
    c = cases.case_vortex(21, 15, 10)
    g, o = pair(c, i_end=21)
    _steps(g, o, 15, graph=graph)
    assert max(per_var_rel_linf(g.get_conservative(), o.get_conservative())) <= 1e-10
    g, o = pair(c, viscous=True, Re=200.0, i_end=21)
    _steps(g, o, 15, graph=graph)
    assert max(per_var_rel_linf(g.get_conservative(), o.get_conservative())) <= 1e-10
    prim_g, prim_o = g.get_primitive(), o.get_primitive()
    assert rel_linf(prim_g[5], prim_o[5]) <= 1e-10  # temperature incl. ghost layers


def test_steps_naca_freestream_viscous():
    c = cases.case_naca(48, 24, 6, first=1e-3)
    g, o = pair(c)
    _steps(g, o, 10, graph=True)
    assert max(per_var_rel_linf(g.get_conservative(), o.get_conservative())) <= 1e-10


def test_short_dimension_extension():
    """KM = 4: the reference's stencils would index outside the grid; both
    implementations use the 2nd-order extension for the metrics."""
    c = cases.case_naca(40, 20, 4, first=1e-3)
    g, o = pair(c)
    # the stretched O-grid's metrics come from differences of nearly equal
    # coordinates; FMA contraction on the GPU moves them by ~1e-12 relative
    assert rel_linf(g.get_metrics(), o.get_metrics()) <= 1e-10
    _steps(g, o, 5, graph=True)
    assert max(per_var_rel_linf(g.get_conservative(), o.get_conservative())) <= 1e-10


def test_t_end_clamp_and_finish():
    c = cases.case_vortex(20, 14, 10)
    g, o = pair(c)
    dt0 = o.calc_dt()
    t_end = 2.5 * dt0
    g.set_time(0.0)
    done = g.run(10, t_end)
    rc, to, no = o.solve(10, t_end)
    assert done == no == 3
    t, _ = g.get_time()
    assert abs(t - to) <= 1e-14 and abs(t - t_end) <= 1e-12
    assert max(per_var_rel_linf(g.get_conservative(), o.get_conservative())) <= 1e-11


def test_split_precision_accuracy():
    c = cases.case_vortex(64, 32, 16)
    g, o = pair(c, precision=PREC_SPLIT)
    _steps(g, o, 50, graph=True)
    rg = interior(g.get_conservative(), c.shape)[..., 0]
    ro = interior(o.get_conservative(), c.shape)[..., 0]
    l2 = np.sqrt(np.mean((rg - ro) ** 2)) / np.sqrt(np.mean(ro ** 2))
    assert l2 <= 1e-5, l2
    assert l2 > 0  # really a different arithmetic


def test_split_precision_accuracy_viscous():
    """Viscous, split precision: the node fluxes and their divergence are held
    in FP32 like the inviscid flux; the state stays within the FP32 flux's
    error of the FP64 oracle (Re 100 makes the viscous terms count)."""
    c = cases.case_vortex(48, 24, 12)
    g, o = pair(c, precision=PREC_SPLIT, viscous=True, Re=100.0)
    _steps(g, o, 30, graph=True)
    for n in (0, 1, 2, 4):  # the w momentum of this quasi-2D flow is round-off sized
        vg = interior(g.get_conservative(), c.shape)[..., n]
        vo = interior(o.get_conservative(), c.shape)[..., n]
        l2 = np.sqrt(np.mean((vg - vo) ** 2)) / max(np.sqrt(np.mean(vo ** 2)), 1e-30)
        assert l2 <= 1e-5, (n, l2)


def test_deterministic():
    c = cases.case_vortex(37, 23, 9)
    outs = []
    for _ in range(2):
        g, _o = pair(c)
        g.set_time(0.0)
        g.run(5)
        outs.append(g.get_conservative())
    assert np.array_equal(outs[0], outs[1])


def test_nan_dt_is_reported_not_thrown():
    c = cases.case_vortex(20, 14, 10)
    Q = c.Q0.copy()
    Q[5, 7, 9, 4] = -10.0  # negative energy -> negative pressure -> NaN sound speed
    g = Block(make_params(*c.shape, **c.params))
    g.calc_metrics(c.x, c.y, c.z)
    g.set_conservative(Q)
    g.set_bc_calc_primitive(CBNS_Q)
    with pytest.raises(CbnsError) as e:
        g.calc_dt()
    assert e.value.code == CBNS_ERR_NAN_DT
    g.set_time(0.0)
    with pytest.raises(CbnsError) as e:
        g.run(3)
    assert e.value.code == CBNS_ERR_NAN_DT


def test_gradient_known_answer():
    from cbns3d_cuda_b200 import calc_gradient
    k, j, i = np.meshgrid(np.arange(150.0), np.arange(100.0), np.arange(50.0), indexing="ij")
    fx, fy, fz = calc_gradient(i * i + j * j + k * k)
    assert max(np.abs(fx - 2 * i).max(), np.abs(fy - 2 * j).max(), np.abs(fz - 2 * k).max()) <= 1e-5
    fx, fy, fz = calc_gradient(i * j * k)
    assert max(np.abs(fx - j * k).max(), np.abs(fy - i * k).max(), np.abs(fz - i * j).max()) <= 1e-5
