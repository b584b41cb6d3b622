"""The per-call path (the reference's own time loop through the C ABI):

* after an inviscid stage 3 and set_bc_calc_primitive(Q), calc_dt reads the
  spectral-radius maximum those two calls accumulated; it equals the maximum
  of a full sweep over the same state;
* a hybrid context evaluates the sensor on the first stage-1 call and on
  every sensor_interval-th one after it, the decisions holding in between,
  and counts the steps so that the audit's rotating sample advances as in a
  run: per-call steps follow cbns_run's schedule, to the same decisions and
  the same state, bit for bit.
"""
from pathlib import Path

import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, PREC_FP64, PREC_HYBRID, Block, cases, make_params

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz"


def _block(case, precision):
    b = Block(make_params(*case.shape, **case.params, precision=precision))
    b.calc_metrics(case.x, case.y, case.z)
    b.set_conservative(case.Q0)
    b.set_bc_calc_primitive(CBNS_Q)
    if precision == PREC_HYBRID:
        w = np.load(WEIGHTS)
        b.sensor_load(w["params"].astype(np.float32), float(w["tau"]))
    return b


def test_calc_dt_reads_the_accumulated_radius():
    c = cases.case_shock_vortex(48, 40, 16)
    g = _block(c, PREC_FP64)
    t = 0.0
    for _ in range(3):
        t = g.step_like_reference(t, 1.0e30)
    dt_acc = g.calc_dt()  # from stage 3 and the boundary update of the last step
    g.set_conservative(g.get_conservative())  # the same state, now without an accumulated radius
    g.set_bc_calc_primitive(CBNS_Q)
    dt_sweep = g.calc_dt()
    assert dt_acc > 0.0
    assert abs(dt_acc - dt_sweep) <= 1e-14 * dt_sweep


def test_percall_sensor_follows_the_run_schedule():
    c = cases.case_shock_vortex(48, 40, 16)
    a = _block(c, PREC_HYBRID)
    b = _block(c, PREC_HYBRID)
    a.sensor_interval(3)
    b.sensor_interval(3)
    masks = []
    t = 0.0
    for _ in range(5):
        t = a.step_like_reference(t, 1.0e30)
        masks.append(a.sensor_mask()[0].copy())
    # steps 2 and 3 hold the decisions of step 1; step 4 evaluates again
    assert np.array_equal(masks[0], masks[1]) and np.array_equal(masks[0], masks[2])
    assert not np.array_equal(masks[2], masks[3])
    assert np.array_equal(masks[3], masks[4])
    b.set_time(0.0)
    assert b.run(5) == 5
    assert np.array_equal(b.sensor_mask()[0], masks[4])
    assert np.array_equal(a.get_conservative(), b.get_conservative())
    assert b.get_time()[0] == t
    sa, sb = a.sensor_stats(), b.sensor_stats()
    assert sa["audit_faces"] == sb["audit_faces"] and sa["audit_fail_steps"] == sb["audit_fail_steps"]
