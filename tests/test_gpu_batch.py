"""Batches (cbns_batch_*): independent blocks advanced together by one
persistent work-queue launch of the stage kernel per RK stage.

The batch computes what each block computes alone — the same stage arithmetic,
boundary conditions and per-block time step — so after several steps every
block's state and time equal those of the block run by itself: bit for bit for
the plain (FP64) path (the block alone on the synchronously staged variant,
as the batched FP64 kernel stages); for the split and hybrid paths the state agrees to the
FP32 rounding of the flux, and the hybrid's sensor decisions agree but for
faces at the threshold (the batched stage and sensor kernels are separate
compilations of the same source, free to contract their FP32 products into
fused multiply-adds differently).
"""
from pathlib import Path

import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, PREC_FP64, PREC_HYBRID, PREC_SPLIT, Batch, Block, cases, make_params
from cbns3d_cuda_b200._abi import CbnsError
from tests.helpers import per_var_rel_linf

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz"


def _block(case, precision, nudge=0.0):
    p = dict(case.params)
    b = Block(make_params(*case.shape, **p, precision=precision))
    if precision == PREC_FP64:
        b.stage_variant(0)  # the batched FP64 kernel stages each plane synchronously
    b.calc_metrics(case.x, case.y, case.z)
    b.set_conservative(case.Q0)
    if p.get("viscous"):
        b.calc_primitive(CBNS_Q)
    b.set_bc_calc_primitive(CBNS_Q)
    if p.get("viscous"):
        b.calc_viscous_terms()
    if precision == PREC_HYBRID:
        w = np.load(WEIGHTS)
        params = w["params"].astype(np.float32)
        params[-1] += np.float32(nudge)  # the output bias: another network
        b.sensor_load(params, float(w["tau"]))
    b.set_time(0.0)
    return b


# bc_mode 1 (far field on every face, the batched-block configuration's) runs
# the blocks' boundary and viscous node kernels as one batched launch each per
# stage; bc_mode 0 (the reference's boundaries) runs them block by block.  The
# hybrid's sensor kernels run batched when every block carries the same
# network, block by block otherwise (mixed: block 0 gets another network).
@pytest.mark.parametrize("precision,viscous,bc_mode,mixed",
                         [(PREC_FP64, False, 1, False), (PREC_SPLIT, False, 1, False), (PREC_SPLIT, True, 1, False),
                          (PREC_FP64, True, 1, False), (PREC_HYBRID, False, 1, False), (PREC_HYBRID, True, 1, False),
                          (PREC_HYBRID, True, 1, True), (PREC_HYBRID, False, 0, False), (PREC_FP64, True, 0, False),
                          (PREC_SPLIT, False, 0, False)])
def test_batch_equals_blocks_alone(precision, viscous, bc_mode, mixed):
    cs, draw = cases.case_batch(5, seed=3, size_lo=(20, 14, 10), size_hi=(44, 30, 18), viscous=viscous)
    for c in cs:
        c.params["bc_mode"] = bc_mode
    n = 8
    nudges = [0.25 if (mixed and i == 0) else 0.0 for i in range(len(cs))]
    alone = [_block(c, precision, u) for c, u in zip(cs, nudges)]
    for b in alone:
        assert b.run(n) == n
    together = [_block(c, precision, u) for c, u in zip(cs, nudges)]
    with Batch(together) as bt:
        assert bt.run(n) == n
        assert bt.run(2) == 2  # the captured step replays
    for b in alone:
        assert b.run(2) == 2
    times = []
    for a, b in zip(alone, together):
        qa, qb = a.get_conservative(), b.get_conservative()
        ta, tb = a.get_time()[0], b.get_time()[0]
        if precision in (PREC_HYBRID, PREC_SPLIT):
            if precision == PREC_HYBRID:
                ma, mb = a.sensor_mask()[0], b.sensor_mask()[0]
                assert np.mean(ma != mb) <= 1e-3  # a face at the threshold may flip
            # relative to the whole state (the w momentum of these quasi-2D
            # flows is round-off sized, so per-variable ratios mean nothing)
            assert np.max(np.abs(qb - qa)) <= 1e-6 * np.max(np.abs(qa))
            assert per_var_rel_linf(qb, qa)[0] <= 1e-6
            assert abs(ta - tb) <= 1e-6 * ta
        else:
            assert np.array_equal(qa, qb)
            assert ta == tb
        times.append(ta)
    assert len(set(times)) == len(times)  # each block its own dt


def test_batch_rejects_mixed_blocks():
    cs, _ = cases.case_batch(2, seed=4, size_lo=(20, 14, 10), size_hi=(24, 16, 12), viscous=False)
    a = _block(cs[0], PREC_SPLIT)
    b = _block(cs[1], PREC_FP64)
    with pytest.raises(CbnsError):
        Batch([a, b])
    with pytest.raises(CbnsError):
        Batch([a, a])
    c = Block(make_params(*cs[1].shape, **cs[1].params, precision=PREC_SPLIT))  # no metrics yet
    with pytest.raises(CbnsError):
        Batch([a, c])


def test_batch_follows_block_settings():
    """A setting changed on a block after the batch captured its step (here the
    sensor's network interval, which sets the widening width) reaches the
    batch's next run: the batch captures the step anew."""
    cs, _ = cases.case_batch(3, seed=5, size_lo=(20, 14, 10), size_hi=(36, 24, 16), viscous=False)
    alone = [_block(c, PREC_HYBRID) for c in cs]
    together = [_block(c, PREC_HYBRID) for c in cs]
    for b in alone:
        assert b.run(4) == 4
        b.sensor_interval(1)
        assert b.run(3) == 3
    with Batch(together) as bt:
        assert bt.run(4) == 4
        for b in together:
            b.sensor_interval(1)
        assert bt.run(3) == 3
    for a, b in zip(alone, together):
        ma, mb = a.sensor_mask()[0], b.sensor_mask()[0]
        assert np.mean(ma != mb) <= 1e-3
        qa, qb = a.get_conservative(), b.get_conservative()
        assert np.max(np.abs(qb - qa)) <= 1e-6 * np.max(np.abs(qa))
