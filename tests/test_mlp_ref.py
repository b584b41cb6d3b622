"""The numpy restatement of the sensor network's gradient (the checker of the
GPU backward kernel) against central finite differences of its own loss."""
import numpy as np

from cbns3d_cuda_b200 import sensor
from oracle import mlp_ref


def test_numpy_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((50, 15))
    Y = (rng.random(50) < 0.4).astype(np.uint8)
    P = sensor.init_params(2).astype(np.float64)
    P[480:512] = 0.1
    P[1536:1568] = 0.05
    _, g = mlp_ref.loss_grad(P, X, Y, 2.0)
    idx = np.arange(0, 1601, 23)
    num = np.empty(len(idx))
    h = 1e-6
    for n, i in enumerate(idx):
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        num[n] = (mlp_ref.loss_grad(Pp, X, Y, 2.0)[0] - mlp_ref.loss_grad(Pm, X, Y, 2.0)[0]) / (2 * h)
    assert np.max(np.abs(num - g[idx])) <= 1e-6 * np.max(np.abs(g[idx]))
