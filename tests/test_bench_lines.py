"""Host logic of bench.py's lines, on the CPU: both arms describe the same
workload in `config`, and the reference arm's per-step time keeps the
shortest run of each step count (its first run carries start-up time)."""
import pytest

import bench
from cbns3d_cuda_b200 import cases


def test_both_arms_share_the_workload_config():
    c = cases.case_vortex(20, 14, 10)
    a = bench.workload_config("shock-vortex 20x14x10", c, 1234)
    b = bench.workload_config("shock-vortex 20x14x10", c, 1234)
    assert a == b
    assert set(a) == {"workload", "grid", "cell_updates_per_step", "l2"}
    assert a["grid"] == [20, 14, 10] and a["cell_updates_per_step"] == 1234


def test_reference_time_keeps_the_shortest_runs():
    # a measured pair: the first 5-step run carried 0.76 s of start-up time
    runs = {5: [0.957142, 0.193793], 25: [1.08846, 0.903808]}
    sec = bench.ref_loop_seconds(runs, 5, 20)
    assert sec == pytest.approx(0.903808 - 0.193793)
    assert 1e3 * sec / 20 == pytest.approx(35.50, abs=0.01)
    # never zero or negative
    assert bench.ref_loop_seconds({3: [2.0], 5: [1.0]}, 3, 2) == pytest.approx(1e-9)
