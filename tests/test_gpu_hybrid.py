"""The hybrid flux (precision PREC_HYBRID) through the C ABI.

* a sensor that sends every face to WENO5 reproduces the split path bit for bit;
* the GPU's own decisions (read back with cbns_sensor_mask_get) given to the
  oracle's hybrid flux reproduce the GPU right-hand side and steps to the
  accuracy of the split path's FP32 flux arithmetic;
* the audit catches a sensor that sends shock faces to the linear flux and
  the step then equals the all-WENO5 step;
* a hybrid context refuses to step before its sensor is loaded.
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, PREC_HYBRID, PREC_SPLIT, Block, cases, make_params
from cbns3d_cuda_b200._abi import CBNS_ERR_STATE, CbnsError
from oracle import oracle as orc
from tests.helpers import interior, per_var_rel_linf

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from cbns3d_cuda_b200 import sensor  # noqa: E402


def _setup(b, case):
    b.calc_metrics(case.x, case.y, case.z)
    b.set_conservative(case.Q0)
    b.set_bc_calc_primitive(CBNS_Q)
    return b


def _block(case, precision, params=None, tau=0.5, audit=(97, 1.0e-2)):
    b = _setup(Block(make_params(*case.shape, **case.params, precision=precision)), case)
    if precision == PREC_HYBRID:
        b.sensor_load(params, tau)
        b.sensor_audit(*audit)
    return b


def _oracle(case):
    return _setup(orc.OracleBlock(make_params(*case.shape, **case.params)), case)


def _constant_sensor(logit):
    """A network whose output logit is the constant `logit` (all weights zero)."""
    P = np.zeros(sensor.NPARAM, dtype=np.float32)
    P[sensor.P_B3] = logit
    return P


def _jump_sensor(block):
    """A hand-built network with logit = (sum_m |f_m| - cut) / cut: the first
    layer forms relu(f_m) and relu(-f_m), the second sums them.  cut is the
    median of sum |f| over the block's faces with a non-zero sum, so that
    faces in uniform flow and the weaker half of the others take the linear
    flux and the rest WENO5."""
    P = np.zeros(sensor.NPARAM, dtype=np.float32)
    for m in range(sensor.NIN):
        P[sensor.P_W1 + (2 * m) * sensor.NIN + m] = 1.0
        P[sensor.P_W1 + (2 * m + 1) * sensor.NIN + m] = -1.0
    P[sensor.P_W2:sensor.P_W2 + 2 * sensor.NIN] = 1.0  # row 0 of W2
    X, _ = sensor.sample_faces(block)
    s = np.abs(X.cpu().numpy().astype(np.float64)).sum(axis=1)
    cut = float(np.median(s[s > 0]))
    P[sensor.P_W3] = 1.0 / cut
    P[sensor.P_B3] = -1.0
    return P


def _both_used(m):
    n1 = int(m.sum())
    return n1 >= 100 and m.size - n1 >= 100


SMALL = [lambda: cases.case_blast(24, 24, 24), lambda: cases.case_shock_vortex(40, 36, 12)]


@pytest.mark.parametrize("make", SMALL)
def test_all_weno_sensor_equals_split(make):
    c = make()
    s = _block(c, PREC_SPLIT)
    h = _block(c, PREC_HYBRID, _constant_sensor(30.0))
    for b in (s, h):
        b.set_time(0.0)
        assert b.run(6) == 6
    assert np.array_equal(h.get_conservative(), s.get_conservative())
    st = h.sensor_stats()
    assert st["weno_faces"] == 6 * st["faces_per_step"]
    assert st["audit_faces"] == 0 and st["audit_fail_steps"] == 0 and st["sensor_fail"] == 0
    m, forced = h.sensor_mask()
    assert np.all(m == 1) and not forced


@pytest.mark.parametrize("make", SMALL)
def test_rhs_matches_oracle_under_gpu_decisions(make):
    c = make()
    s = _block(c, PREC_SPLIT)
    o = _oracle(c)
    if c.name == "blast":  # develop the blast wave first
        s.set_time(0.0)
        s.run(8)
        Q = s.get_conservative()
        o.set_conservative(Q)
        o.set_bc_calc_primitive(CBNS_Q)
    else:
        Q = c.Q0
    err_split = max(per_var_rel_linf(s.eval_rhs(CBNS_Q), o.eval_rhs(CBNS_Q)))
    tol = max(4.0 * err_split, 1.0e-6)  # the split path's FP32 flux arithmetic
    h = _block(c, PREC_HYBRID, _constant_sensor(-30.0), audit=(1, 1.0e30))
    h.set_conservative(Q)
    h.set_bc_calc_primitive(CBNS_Q)
    # every face linear: matches the oracle's linear flux, not its WENO5
    rhs = h.eval_rhs(CBNS_Q)
    m, forced = h.sensor_mask()
    assert not forced and np.all(m == 0)
    o.set_face_mask(m)
    lin_o = o.eval_rhs(CBNS_Q).reshape(-1, 5)
    # at the blast's strong shock the linear reconstruction can reach negative
    # pressure, where the sound speed is NaN (the oracle's wave-speed bound
    # then propagates it, the GPU's fmax drops it): compare the other nodes
    fin = np.all(np.isfinite(lin_o), axis=1)
    assert fin.mean() > 0.9
    rhs2 = rhs.reshape(-1, 5)
    err_lin = max(per_var_rel_linf(rhs2[fin], lin_o[fin]))
    o.set_face_mask(None)
    err_weno = max(per_var_rel_linf(rhs2[fin], o.eval_rhs(CBNS_Q).reshape(-1, 5)[fin]))
    assert err_lin <= tol and err_weno > 100 * err_lin, (err_lin, err_weno, err_split)
    # a mixture of both fluxes
    h.sensor_load(_jump_sensor(h), 0.5)
    rhs = h.eval_rhs(CBNS_Q)
    m, forced = h.sensor_mask()
    assert not forced and _both_used(m), m.mean()
    o.set_face_mask(m)
    err = max(per_var_rel_linf(rhs, o.eval_rhs(CBNS_Q)))
    assert err <= tol, (err, err_split)


def test_steps_match_oracle_under_gpu_decisions():
    c = cases.case_shock_vortex(40, 36, 12)
    h = _block(c, PREC_HYBRID, _constant_sensor(0.0), audit=(1, 1.0e30))
    h.sensor_load(_jump_sensor(h), 0.5)
    o = _oracle(c)
    h.set_time(0.0)
    for _ in range(10):
        assert h.run(1) == 1
        m, forced = h.sensor_mask()
        assert not forced and _both_used(m)
        o.set_face_mask(m)
        rc, _t, n = o.solve(1, 1e30)
        assert rc == 0 and n == 1
    rg = interior(h.get_conservative(), c.shape)[..., 0]
    ro = interior(o.get_conservative(), c.shape)[..., 0]
    l2 = np.sqrt(np.mean((rg - ro) ** 2)) / np.sqrt(np.mean(ro ** 2))
    assert 0 < l2 <= 1e-5, l2


def test_audit_forces_weno():
    c = cases.case_shock_vortex(40, 36, 12)
    s = _block(c, PREC_SPLIT)
    # every face linear, every linear face audited, tight bound: the shock trips it
    h = _block(c, PREC_HYBRID, _constant_sensor(-30.0), audit=(1, 1.0e-3))
    for b in (s, h):
        b.set_time(0.0)
        assert b.run(4) == 4
    st = h.sensor_stats()
    assert st["weno_faces"] == 0
    assert st["audit_fail_steps"] == 4 and st["audit_max"] > 1.0e-3
    assert st["audit_faces"] == 4 * st["faces_per_step"]
    m, forced = h.sensor_mask()
    assert forced and np.all(m == 0)
    assert np.array_equal(h.get_conservative(), s.get_conservative())


def test_audit_rotating_sample_and_pass():
    c = cases.case_vortex(20, 14, 10)
    h = _block(c, PREC_HYBRID, _constant_sensor(-30.0), audit=(7, 1.0e30))
    h.set_time(0.0)
    assert h.run(7) == 7
    st = h.sensor_stats()
    # over 7 consecutive steps the rotating offset visits every residue once
    assert st["audit_faces"] == st["faces_per_step"]
    assert st["audit_fail_steps"] == 0
    h.sensor_stats_reset()
    assert h.sensor_stats()["audit_faces"] == 0


def test_hybrid_needs_sensor_and_rejects_bad_arguments():
    c = cases.case_vortex(20, 14, 10)
    h = _setup(Block(make_params(*c.shape, **c.params, precision=PREC_HYBRID)), c)
    h.set_time(0.0)
    with pytest.raises(CbnsError) as e:
        h.run(1)
    assert e.value.code == CBNS_ERR_STATE
    with pytest.raises(CbnsError):
        h.sensor_load(_constant_sensor(0.0), 1.5)
    bad = _constant_sensor(0.0)
    bad[3] = np.nan
    with pytest.raises(CbnsError):
        h.sensor_load(bad, 0.5)
    with pytest.raises(CbnsError):
        h.sensor_audit(0, 1e-2)
    s = _setup(Block(make_params(*c.shape, **c.params, precision=PREC_SPLIT)), c)
    with pytest.raises(CbnsError) as e:
        s.sensor_load(_constant_sensor(0.0), 0.5)
    assert e.value.code == CBNS_ERR_STATE
