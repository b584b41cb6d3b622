"""TMA staging of the stage kernel.

The plain FP64 stage kernel has two compiled variants with the same
arithmetic: variant 0 stages each plane with synchronous loads, variant 1 by
TMA (ring column, plane with halo and area vectors as 4-D box copies on an
mbarrier).  Both must give the same state bit for bit -- inviscid and viscous,
graph-replayed and per-call steps, single right-hand sides, tiles cut by the
grid's edge in i, j and k.  (The FP32 kernels stage their halo and area
vectors by TMA in every 2- and 3-CTA variant; their results are held to the
oracle by the split-precision and hybrid tests.)
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, PREC_FP64, Block, cases, make_params

pytestmark = pytest.mark.gpu

CASES = {
    # partial tiles: IM-2 and JM-2 not multiples of 16 and 15
    "vortex_partial": lambda: cases.case_vortex(45, 37, 19),
    "vortex_c0": lambda: cases.case_vortex(64, 32, 16),
    "shock_vortex": lambda: cases.case_shock_vortex(70, 50, 12),
    "naca_viscous": lambda: cases.case_naca(48, 24, 6, first=1e-3),
}


def _block(c, variant):
    p = dict(c.params)
    b = Block(make_params(*c.shape, **p, precision=PREC_FP64))
    assert b.stage_variant() == 2
    b.stage_variant(variant)
    b.calc_metrics(c.x, c.y, c.z)
    if c.Q0 is None:
        b.initial_condition()
        b.calc_conservative(CBNS_Q)
    else:
        b.set_conservative(c.Q0)
        if p.get("viscous"):
            b.calc_primitive(CBNS_Q)
    b.set_bc_calc_primitive(CBNS_Q)
    if p.get("viscous"):
        b.calc_viscous_terms()
    b.set_time(0.0)
    return b


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_tma_variant_equals_synchronous(name):
    c = CASES[name]()
    out = []
    for v in (0, 1):
        b = _block(c, v)
        r0 = b.eval_rhs(CBNS_Q)
        assert b.run(7) == 7
        t = b.get_time()[0]
        for _ in range(2):  # per-call steps after the graph-replayed ones
            t = b.step_like_reference(t, 1.0e30)
        out.append((r0, b.get_conservative(), t))
        b.close()
    (ra, qa, ta), (rb, qb, tb) = out
    assert np.all(np.isfinite(qa)) and np.all(np.isfinite(qb))
    d = np.flatnonzero(ra != rb)
    detail = (f"{d.size} of {ra.size} right-hand-side values differ; max relative difference "
              f"{np.max(np.abs(ra - rb)) / np.max(np.abs(ra)):.3e}; first {d[:8].tolist()}")
    assert np.array_equal(ra, rb), detail
    assert np.array_equal(qa, qb)
    assert ta == tb


def test_stage_variant_arguments():
    c = cases.case_vortex(20, 14, 10)
    b = Block(make_params(*c.shape, **c.params, precision=PREC_FP64))
    assert b.stage_variant() == 2
    from cbns3d_cuda_b200._abi import CbnsError
    with pytest.raises(CbnsError):
        b.stage_variant(2)
    b.close()
