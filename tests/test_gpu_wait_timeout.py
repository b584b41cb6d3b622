"""The time-out path of the library's bounded waits, exercised without a fault.

Every wait of the GPU code on an mbarrier -- the sensor's tensor-core MMA
completion (two bounded windows, then the step takes WENO5 everywhere) and the
stage kernel's TMA plane staging (then the state is reported invalid) -- has
an iteration limit.  Here one thread waits on barriers that nothing
completes, through the same wait routines: both report a time-out within a
few seconds, and the device then runs a step as before.
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import Block, cases, make_params, selftest_waits

pytestmark = pytest.mark.gpu


def test_bounded_waits_time_out_and_report():
    r = selftest_waits()
    assert r["mma_timed_out"] == 1 and r["tma_timed_out"] == 1
    # bounded by the iteration limits (measured 4.2 s per window on a B200;
    # two windows for the MMA wait)
    assert 0.0 < r["mma_seconds"] < 40.0 and 0.0 < r["tma_seconds"] < 20.0
    # the context is still usable
    c = cases.case_vortex(20, 14, 10)
    b = Block(make_params(*c.shape, **c.params))
    b.calc_metrics(c.x, c.y, c.z)
    b.set_conservative(c.Q0)
    b.set_bc_calc_primitive()
    b.set_time(0.0)
    assert b.run(2) == 2
    assert np.all(np.isfinite(b.get_conservative()))
    b.close()
