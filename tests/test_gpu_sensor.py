"""The learned shock sensor's kernels against CPU restatements.

* face features and WENO-weight deviation (FP32 on the GPU) vs the oracle's
  FP64 restatement (orc_sensor_faces), face by face;
* the hand-written forward/backward kernel vs a numpy FP64 gradient;
* Adam training lowers the loss;
* tcgen05 BF16 inference vs FP32 inference.
"""
import numpy as np
import pytest

from cbns3d_cuda_b200 import CBNS_Q, Block, cases, make_params
from oracle import mlp_ref
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from cbns3d_cuda_b200 import sensor  # noqa: E402


def _blocks(case, steps=0):
    IM, JM, KM = case.shape
    g = Block(make_params(IM, JM, KM, **case.params))
    o = orc.OracleBlock(make_params(IM, JM, KM, **case.params))
    for b in (g, o):
        b.calc_metrics(case.x, case.y, case.z)
        b.set_conservative(case.Q0)
        b.set_bc_calc_primitive(CBNS_Q)
    if steps:
        g.set_time(0.0)
        g.run(steps)
        o.set_conservative(g.get_conservative().reshape(-1))
    return g, o


@pytest.mark.parametrize("make,steps", [(lambda: cases.case_vortex(20, 14, 10), 0),
                                        (lambda: cases.case_blast(24, 24, 24), 12)])
def test_features_and_labels_match_oracle(make, steps):
    g, o = _blocks(make(), steps)
    feat, lab, dev, idx = sensor.sample_faces(g, with_dev=True)
    f_ref, d_ref = o.sensor_faces(CBNS_Q)
    idx = idx.cpu().numpy()
    assert len(idx) == len(d_ref) and np.array_equal(np.sort(idx), np.arange(len(d_ref)))
    f = feat.cpu().numpy()
    d = dev.cpu().numpy()
    fr, dr = f_ref[idx], d_ref[idx]
    assert np.max(np.abs(f - fr)) <= 1e-4 * max(1.0, np.max(np.abs(fr)))
    assert np.max(np.abs(d - dr)) <= 2e-3
    clear = np.abs(dr - 0.05) > 5e-3
    assert np.array_equal(lab.cpu().numpy()[clear], (dr[clear] > 0.05).astype(np.uint8))


def test_gradient_matches_numpy():
    rng = np.random.default_rng(3)
    n = 1000
    X = rng.standard_normal((n, 15)).astype(np.float32)
    Y = (rng.random(n) < 0.3).astype(np.uint8)
    P = sensor.init_params(5)
    P[480:512] = 0.1 * rng.standard_normal(32)
    P[1536:1568] = 0.1 * rng.standard_normal(32)
    loss, g = sensor.loss_and_grad(torch.from_numpy(P).cuda(), torch.from_numpy(X).cuda(),
                                   torch.from_numpy(Y).cuda(), pos_weight=2.5)
    l_ref, g_ref = mlp_ref.loss_grad(P, X, Y, pos_weight=2.5)
    assert abs(float(loss.item()) - l_ref) <= 1e-4 * abs(l_ref)
    g = g.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(g - g_ref)) <= 1e-4 * np.max(np.abs(g_ref))


def test_training_lowers_loss():
    rng = np.random.default_rng(4)
    n = 20000
    X = rng.standard_normal((n, 15)).astype(np.float32)
    Y = ((X[:, 2] ** 2 + X[:, 7] ** 2) > 1.5).astype(np.uint8)  # a separable target
    Xd, Yd = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
    P, hist = sensor.train(Xd, Yd, epochs=30, batch=2048, lr=3e-3, pos_weight=1.0)
    assert hist[-1] < 0.5 * hist[0]
    p = sensor.predict(P, Xd).cpu().numpy()
    assert np.mean((p > 0.5) == (Y > 0)) > 0.9


def test_tensor_core_inference_matches_fp32():
    rng = np.random.default_rng(6)
    n = 128 * 37 + 19  # several tiles and a partial one
    X = torch.from_numpy(rng.standard_normal((n, 15)).astype(np.float32)).cuda()
    P = torch.from_numpy(sensor.init_params(7)).cuda()
    p32 = sensor.predict(P, X, tensor_cores=False).cpu().numpy()
    ptc = sensor.predict(P, X, tensor_cores=True).cpu().numpy()
    assert np.all(np.isfinite(ptc))
    # BF16 operands (8 significant bits), FP32 accumulation
    assert np.max(np.abs(ptc - p32)) <= 0.03
    assert np.mean(np.abs(ptc - p32)) <= 3e-3
