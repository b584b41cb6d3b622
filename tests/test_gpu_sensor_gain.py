"""What the trained sensor gains over the method without it.

On the shock / vortex grid of 256 x 256 x 128, 30 steps from the initial state:
the split-precision path (every face WENO5, FP32 flux) against the hybrid with
the committed network.  The hybrid must stay within the density L2 bound of the
plain FP64 path (1e-5) while sending most faces to the linear flux, and its
step must be faster than the split path's (device time of the whole step,
sensor and audit included, CUDA events on the launch stream).
"""
from pathlib import Path

import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, PREC_FP64, PREC_HYBRID, PREC_SPLIT, Block, cases, make_params
from tests.helpers import interior

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

WEIGHTS = Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz"


def _run(case, precision, nsteps, sensor=None):
    b = Block(make_params(*case.shape, **case.params, precision=precision))
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    b.calc_metrics(case.x, case.y, case.z)
    b.set_conservative(case.Q0)
    b.set_bc_calc_primitive(CBNS_Q)
    if sensor is not None:
        b.sensor_load(*sensor)
    b.autotune()
    b.set_time(0.0)
    assert b.run(2) == 2  # first-call costs and graph capture
    if sensor is not None:
        b.sensor_stats_reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    b.run_async(nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nsteps
    rho = interior(b.get_conservative(), case.shape)[..., 0].copy()
    stats = b.sensor_stats() if sensor is not None else None
    b.close()
    return ms, rho, stats


def test_trained_sensor_gain_over_split_path():
    w = np.load(WEIGHTS)
    sensor = (w["params"].astype(np.float32), float(w["tau"]))
    c = cases.case_shock_vortex(256, 256, 128)
    n = 30
    _, r64, _ = _run(c, PREC_FP64, n)
    ms32, r32, _ = _run(c, PREC_SPLIT, n)
    msh, rh, st = _run(c, PREC_HYBRID, n, sensor)

    def l2(r):
        return float(np.sqrt(np.mean((r - r64) ** 2) / np.mean(r64 ** 2)))

    weno = st["weno_faces"] / (n * st["faces_per_step"])
    print(f"split {ms32:.3f} ms/step (rho-L2 {l2(r32):.2e}); hybrid {msh:.3f} ms/step (rho-L2 {l2(rh):.2e}), "
          f"WENO5 faces {weno:.3f}, audit-rejected steps {st['audit_fail_steps']}")
    assert l2(rh) <= 1e-5
    assert weno <= 0.35
    assert st["sensor_fail"] == 0
    assert msh < 0.95 * ms32
