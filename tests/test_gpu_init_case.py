"""cbns_init_case: the configurations' initial states formed on the device
equal those cases.py forms on the host (ghost layers included) to the
rounding of exp/pow (1e-13 relative)."""
import numpy as np
import pytest

from cbns3d_cuda_b200 import Block, cases, make_params
from cbns3d_cuda_b200._abi import CASE_BLAST, CASE_SHOCK_VORTEX, CASE_VORTEX, CbnsError

pytestmark = pytest.mark.gpu


def _device_state(c, kind, prm):
    b = Block(make_params(*c.shape, **c.params))
    b.init_case(kind, c.x, c.y, c.z, prm)
    q = b.get_conservative()
    b.close()
    return q


@pytest.mark.parametrize("make,kind,prm", [
    (lambda: cases.case_vortex(24, 16, 10), CASE_VORTEX, [0.5, 5.0, 3.0, 2.5, 1.0, 1.0, 0.0]),
    (lambda: cases.case_blast(20, 20, 20), CASE_BLAST, [0.01, 10.0, 0.1]),
    (lambda: cases.case_shock_vortex(40, 36, 12), CASE_SHOCK_VORTEX, [1.2, 0.3, 0.075, 0.25, 0.5, 0.5]),
])
def test_device_initial_state_equals_host(make, kind, prm):
    c = make()
    q = _device_state(c, kind, prm).reshape(-1, 5)
    ref = np.asarray(c.Q0).reshape(-1, 5)
    for n in range(5):
        scale = np.max(np.abs(ref[:, n])) or 1.0
        assert np.max(np.abs(q[:, n] - ref[:, n])) <= 1e-13 * scale, n


def test_init_case_rejects_bad_arguments():
    c = cases.case_vortex(12, 10, 8)
    b = Block(make_params(*c.shape, **c.params))
    with pytest.raises(CbnsError):
        b.init_case(7, c.x, c.y, c.z, [0.5])
    with pytest.raises(CbnsError):
        b.init_case(CASE_VORTEX, c.x, c.y, c.z, np.zeros(9))
    b.close()
