"""TMA staging of the stage kernel.

The plain FP64 stage kernel has two compiled variants with the same source
arithmetic: variant 0 stages each plane with synchronous loads, variant 1 by
TMA (ring column, plane with halo and area vectors as 4-D box copies on an
mbarrier).  Both must give the same right-hand sides and states -- inviscid and
viscous, graph-replayed and per-call steps, tiles cut by the grid's edge in i,
j and k -- to the rounding of separate compilations (measured: a few dozen of
~150,000 values differ, by at most 6e-15 relative; the viscous case agrees bit
for bit), so to 1e-13 here.  (The FP32 kernels stage their halo and area
vectors by TMA in every 2- and 3-CTA variant; their results are held to the
oracle by the split-precision and hybrid tests.)
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, PREC_FP64, Block, cases, make_params
from tests.helpers import per_var_rel_linf

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
    assert np.max(np.abs(ra - rb)) <= 1e-13 * np.max(np.abs(ra))
    assert max(per_var_rel_linf(qb, qa)) <= 1e-13
    assert abs(ta - tb) <= 1e-13 * ta


def test_stage_variant_arguments():
    c = cases.case_vortex(20, 14, 10)
    b = Block(make_params(*c.shape, **c.params, precision=PREC_FP64))
    assert b.stage_variant() == 2
    from cbns3d_cuda_b200._abi import CbnsError
    with pytest.raises(CbnsError):
        b.stage_variant(2)
    assert 1 <= b.stage_kchunk() <= 8
    assert b.stage_kchunk(3) == 3 and b.stage_kchunk() == 3
    for bad in (0, 9, -2):
        with pytest.raises(CbnsError):
            b.stage_kchunk(bad)
    b.close()


@pytest.mark.parametrize("variant", [0, 1])
def test_fp64_k_chunk_leaves_results_unchanged(variant):
    """Every chunk computes its planes' fluxes from the same ring of planes,
    so the chunking changes only the work split: the same states bit for bit."""
    c = CASES["vortex_partial"]()
    out = []
    for kc in (-1, 3, 17):
        b = _block(c, variant)
        b.stage_kchunk(kc)
        assert b.run(4) == 4
        out.append((b.get_conservative(), b.get_time()[0]))
        b.close()
    for q, t in out[1:]:
        assert np.array_equal(q, out[0][0]) and t == out[0][1]
