"""The hybrid flux (precision PREC_HYBRID) through the C ABI.

* a sensor that always answers WENO5 follows the split path (flat stencils,
  which take the linear flux without the network, aside);
* the GPU's own decisions (read back with cbns_sensor_mask_get) given to the
  oracle's hybrid flux reproduce the GPU right-hand side and steps to the
  accuracy of the split path's FP32 flux arithmetic;
* the audit catches a sensor that sends shock faces to the linear flux and
  the step then equals the all-WENO5 step (to the FP32 rounding of the flux);
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


FLAT = 0.0045  # sum of |features| below which a stencil is flat (linear flux, no network)


def _flat(X):
    return np.abs(X.cpu().numpy().astype(np.float64)).sum(axis=1) < FLAT


def _widen(dec, shape, along=2, across=1):
    """The library's widening of WENO5 decisions: per face direction, a face
    takes WENO5 when a face of the same direction within `along` faces on its
    own grid line, or `across` faces in the other index directions, does."""
    IM, JM, KM = shape
    ni, nj = (IM - 1) * (JM - 2) * (KM - 2), (IM - 2) * (JM - 1) * (KM - 2)
    # numpy axes (k, j, i); the face direction's own axis
    parts = [(dec[:ni].reshape(KM - 2, JM - 2, IM - 1), 2), (dec[ni:ni + nj].reshape(KM - 2, JM - 1, IM - 2), 1),
             (dec[ni + nj:].reshape(KM - 1, JM - 2, IM - 2), 0)]
    out = []
    for a, own in parts:
        r = a.copy()
        for ax in (2, 1, 0):
            w = along if ax == own else across
            src = r.copy()
            n = src.shape[ax]
            for o in range(1, w + 1):
                lo = [slice(None)] * 3
                hi = [slice(None)] * 3
                lo[ax], hi[ax] = slice(0, n - o), slice(o, n)
                r[tuple(lo)] |= src[tuple(hi)]
                r[tuple(hi)] |= src[tuple(lo)]
        out.append(r.reshape(-1))
    return np.concatenate(out)


@pytest.mark.parametrize("make", SMALL)
def test_always_weno_sensor_matches_split(make):
    """A network that always answers WENO5: every non-flat face takes WENO5,
    flat faces the linear flux, and the state follows the split path to
    within FP32 round-off."""
    c = make()
    s = _block(c, PREC_SPLIT)
    h = _block(c, PREC_HYBRID, _constant_sensor(30.0))
    h.sensor_interval(1)  # fresh decisions every step
    for b in (s, h):
        b.set_time(0.0)
        assert b.run(6) == 6
    rs = interior(s.get_conservative(), c.shape)[..., 0]
    rh = interior(h.get_conservative(), c.shape)[..., 0]
    assert np.sqrt(np.mean((rh - rs) ** 2) / np.mean(rs ** 2)) <= 1e-5
    st = h.sensor_stats()
    assert 0 < st["weno_faces"] <= 6 * st["faces_per_step"]
    assert st["audit_faces"] < st["faces_per_step"] and st["audit_fail_steps"] == 0 and st["sensor_fail"] == 0
    h.eval_rhs(CBNS_Q)
    m, forced = h.sensor_mask()
    X, _y, _d, idx = sensor.sample_faces(h, with_dev=True)
    dec = np.zeros(m.size, np.uint8)
    dec[idx.cpu().numpy()] = ~_flat(X)
    assert not forced and np.array_equal(m, _widen(dec, c.shape))


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


def _check_widened(m, want, near, shape):
    """m equals the widening of want, up to faces whose widened value depends
    on a decision within 1e-4 of the threshold (either answer allowed)."""
    lo = _widen(want & ~near, shape)
    hi = _widen(want | near, shape)
    return bool(np.all((m >= lo) & (m <= hi)))


@pytest.mark.parametrize("make", SMALL + [lambda: cases.case_vortex(37, 23, 9)])
def test_sensor_sweep_matches_sampled_faces(make):
    """The per-step sensor (directional sweeps, tcgen05) decides every face as
    the tensor-core predictor does on the sampled features of the same state."""
    c = make()
    h = _block(c, PREC_HYBRID, _constant_sensor(0.0))
    P = _jump_sensor(h)
    h.sensor_load(P, 0.5)
    h.eval_rhs(CBNS_Q)
    m, _ = h.sensor_mask()
    X, _y, _d, idx = sensor.sample_faces(h, with_dev=True)
    p = sensor.predict(torch.from_numpy(P).cuda(), X, tensor_cores=True).cpu().numpy()
    idx = idx.cpu().numpy()
    assert np.array_equal(np.sort(idx), np.arange(m.size))
    near = np.zeros(m.size, bool)
    near[idx] = np.abs(p - 0.5) < 1e-4  # the sweep tests logit >= logit(tau), here p >= tau
    want = np.zeros(m.size, np.uint8)
    want[idx] = (p >= 0.5) & ~_flat(X)
    assert _check_widened(m, want, near, c.shape)
    assert 0 < m.sum() < m.size


def test_trained_sensor_sweep_matches_sampled_faces():
    """The committed network: the sweep decides every face as the tensor-core
    predictor on the sampled features (flat stencils linear, then widened)."""
    from pathlib import Path
    w = np.load(Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz")
    P, tau = w["params"].astype(np.float32), float(w["tau"])
    c = cases.case_shock_vortex(64, 64, 16)
    h = _block(c, PREC_HYBRID, P, tau)
    h.set_time(0.0)
    assert h.run(5) == 5
    h.eval_rhs(CBNS_Q)
    m, _ = h.sensor_mask()
    X, _y, _d, idx = sensor.sample_faces(h, with_dev=True)
    p = sensor.predict(torch.from_numpy(P).cuda(), X, tensor_cores=True).cpu().numpy()
    idx = idx.cpu().numpy()
    near = np.zeros(m.size, bool)
    near[idx] = np.abs(p - tau) < 1e-4
    want = np.zeros(m.size, np.uint8)
    want[idx] = (p >= tau) & ~_flat(X)
    assert _check_widened(m, want, near, c.shape)
    assert 0 < m.sum() < m.size


def test_uncertain_faces_take_weno():
    """Only faces the committed network is confident are smooth take the linear
    flux: its threshold is at most 0.5 (the network's own decision boundary)
    and keeps the recorded held-out recall floor; scaling a real face's
    features sweeps the network's answer through the uncertainty band [tau,
    0.9); and on a live state every face the predictor places in that band is
    a WENO5 face in the sweep's decisions."""
    import json
    from pathlib import Path
    w = np.load(Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz")
    P, tau = w["params"].astype(np.float32), float(w["tau"])
    summ = json.loads(str(w["summary"]))
    assert tau <= 0.5
    assert summ["val_recall"] >= summ["recall_floor"] >= 0.95
    # crafted features in the band: interpolate between a flat face (p ~ 0) and
    # a strong-jump face (p ~ 1) and keep the points whose p lies in [tau, 0.9)
    c = cases.case_shock_vortex(64, 64, 16)
    h = _block(c, PREC_HYBRID, P, tau)
    X, _ = sensor.sample_faces(h)
    Pt = torch.from_numpy(P).cuda()
    p = sensor.predict(Pt, X, tensor_cores=True)
    hi = X[int(torch.argmax(p))]
    a = torch.linspace(0.0, 1.0, 4096, device="cuda")[:, None]
    Xc = (a * hi[None, :]).contiguous()
    pc = sensor.predict(Pt, Xc, tensor_cores=True).cpu().numpy()
    band = (pc >= tau + 1e-3) & (pc < 0.9)
    # the scaled faces sweep p through the uncertainty band, its lower edge
    # (the network's decision boundary p = 0.5) included
    assert band.sum() >= 10 and np.any((pc >= tau) & (pc < tau + 0.05))
    # the library's decision rule on crafted features: the predictor's p >= tau
    # is WENO5; on the live state the sweep agrees with that rule face by face
    h.eval_rhs(CBNS_Q)
    m, _ = h.sensor_mask()
    Xs, _y, _d, idx = sensor.sample_faces(h, with_dev=True)
    ps = sensor.predict(Pt, Xs, tensor_cores=True).cpu().numpy()
    idx = idx.cpu().numpy()
    in_band = (ps >= tau + 1e-4) & (ps < 0.9) & ~_flat(Xs)
    assert in_band.sum() > 0
    assert np.all(m[idx[in_band]] == 1)


def test_sensor_interval_holds_and_widens_decisions():
    """With the network evaluated every 3rd step, a 3-step run uses the first
    step's decisions, widened by 4 along and 3 across, for all three steps."""
    c = cases.case_shock_vortex(40, 36, 12)
    h = _block(c, PREC_HYBRID, _constant_sensor(0.0), audit=(97, 1.0e30))
    P = _jump_sensor(h)
    h.sensor_load(P, 0.5)
    h.sensor_interval(3)
    X, _y, _d, idx = sensor.sample_faces(h, with_dev=True)  # the initial state
    p = sensor.predict(torch.from_numpy(P).cuda(), X, tensor_cores=True).cpu().numpy()
    idx = idx.cpu().numpy()
    h.sensor_stats_reset()
    h.set_time(0.0)
    assert h.run(3) == 3
    m, forced = h.sensor_mask()
    near = np.zeros(m.size, bool)
    near[idx] = np.abs(p - 0.5) < 1e-4
    want = np.zeros(m.size, np.uint8)
    want[idx] = (p >= 0.5) & ~_flat(X)
    lo, hi = _widen(want & ~near, c.shape, 4, 3), _widen(want | near, c.shape, 4, 3)
    assert not forced and np.all((m >= lo) & (m <= hi))
    assert h.sensor_stats()["weno_faces"] == 3 * int(m.sum())
    with pytest.raises(CbnsError):
        h.sensor_interval(0)


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
    # the forced step runs the split path's flux code (a separate compilation,
    # so equal up to the FP32 rounding of the flux)
    qh, qs = h.get_conservative(), s.get_conservative()
    assert np.max(np.abs(qh - qs)) <= 1e-6 * np.max(np.abs(qs))


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


def test_weights_file_and_driver():
    """cbns_sensor_load_file gives the same decisions as the parameters loaded
    from memory, and the host driver runs the hybrid from its input files."""
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    w = np.load(root / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz")
    c = cases.case_shock_vortex(48, 48, 12)
    a = _block(c, PREC_HYBRID, w["params"].astype(np.float32), float(w["tau"]))
    b = _setup(Block(make_params(*c.shape, **c.params, precision=PREC_HYBRID)), c)
    from cbns3d_cuda_b200 import _abi
    _abi.check(b.lib.cbns_sensor_load_file(b.h, str(root / "cbns3d_cuda_b200" / "data" / "sensor_weights.bin").encode()),
               "cbns_sensor_load_file")
    assert np.array_equal(a.eval_rhs(CBNS_Q), b.eval_rhs(CBNS_Q))
    assert np.array_equal(a.sensor_mask()[0], b.sensor_mask()[0])
    with pytest.raises(CbnsError):
        _abi.check(b.lib.cbns_sensor_load_file(b.h, b"/nonexistent/weights.bin"), "cbns_sensor_load_file")
    exe = root / "cbns3d_cuda_b200" / "bin" / "cbns3d_b200"
    tmp = Path(__import__("tempfile").mkdtemp())
    outs = {}
    for prec in ("fp64", "hybrid"):
        d = c.write(tmp / prec, nsteps=20, checkpoint_freq=20)
        r = subprocess.run([str(exe), "--quiet", "--graph", "--inviscid", "--precision", prec], cwd=d,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        outs[prec] = cases.read_checkpoint(d / "checkpoint.dat")[1]
    r64 = interior(outs["fp64"], c.shape)[..., 0]
    rh = interior(outs["hybrid"], c.shape)[..., 0]
    assert 0 < np.sqrt(np.mean((rh - r64) ** 2) / np.mean(r64 ** 2)) <= 1e-4


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
