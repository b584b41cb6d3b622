"""The reference's own known-answer tests, restated for the oracle.

The reference ships analytic gtest cases for the 4th-order gradient
(test/gradient_test.cpp:20-84 and :86-150, max error <= 1e-5) and for the
metrics (test/metrics_test.cpp: tanh-stretched box MSE <= 2e-2, rotated cube
MSE <= 1e-8, conical shell MSE <= 1e-3).  Inputs are generated here from the
same formulas; the exact Jacobians come from complex-step derivatives of the
mappings.  The same cases run on the GPU in test_gpu_metrics.py.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from cbns3d_cuda_b200 import make_params


def _grid(IM, JM, KM):
    return np.meshgrid(np.arange(KM, dtype=float), np.arange(JM, dtype=float), np.arange(IM, dtype=float),
                       indexing="ij")


def test_gradient_quadratic(oracle_lib):
    IM, JM, KM = 50, 100, 150
    k, j, i = _grid(IM, JM, KM)
    fx, fy, fz = orc.calc_gradient(i * i + j * j + k * k)
    err = max(np.abs(fx - 2 * i).max(), np.abs(fy - 2 * j).max(), np.abs(fz - 2 * k).max())
    assert err <= 1e-5


def test_gradient_product(oracle_lib):
    IM, JM, KM = 50, 100, 150
    k, j, i = _grid(IM, JM, KM)
    fx, fy, fz = orc.calc_gradient(i * j * k)
    err = max(np.abs(fx - j * k).max(), np.abs(fy - i * k).max(), np.abs(fz - i * j).max())
    assert err <= 1e-5


# ---------------------------------------------------------------- metrics
def tanh_box(n=10, L=5.0, s=1.2):
    def f(i, j, k):
        g = lambda t: 0.5 * L * (np.tanh(s * (-1 + 2.0 * t / (n - 1))) + 1)
        return g(i), g(j), g(k)
    return (n, n, n), f


def rotated_cube(n=10, a=np.pi / 4, b=np.pi / 4, c=np.pi / 4):
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    R = np.array([[cb * cc, sa * sb * cc - sc * ca, sa * sc + sb * ca * cc],
                  [sc * cb, sa * sb * sc + ca * cc, -sa * cc + sb * sc * ca],
                  [-sb, sa * cb, ca * cb]])

    def f(i, j, k):
        v = np.stack([i / (n - 1), j / (n - 1), k / (n - 1)])
        return tuple(np.tensordot(R, v, axes=1))
    return (n, n, n), f


def conical_shell(nx=10, ny=20, nz=5, Rx=3.0, Ry=6.0, Rz=5.0, th=5 * np.pi / 12, ph=np.pi / 12):
    def f(i, j, k):
        r = lambda R0: R0 - (R0 - 1.0) * i / (nx - 1)
        a = th * (2.0 * j / (ny - 1) - 1.0)
        b = ph * (2.0 * k / (nz - 1) + 1.0)
        return r(Rx) * np.cos(a) * np.sin(b), r(Ry) * np.sin(a) * np.sin(b), r(Rz) * np.cos(b)
    return (nx, ny, nz), f


def exact_metrics(shape, f):
    """J and the 9 inverse metrics from complex-step derivatives of the map."""
    IM, JM, KM = shape
    k, j, i = _grid(IM, JM, KM)
    h = 1e-30
    cols = []
    for d in range(3):
        args = [i.astype(complex), j.astype(complex), k.astype(complex)]
        args[d] = args[d] + 1j * h
        cols.append(np.stack([c.imag / h for c in f(*args)]))  # d(x,y,z)/d(index_d)
    A = np.stack(cols, axis=1)  # A[r, c] = d x_r / d idx_c
    A = np.moveaxis(A, (0, 1), (-2, -1))
    J = np.linalg.det(A)
    B = np.linalg.inv(A)  # rows: grad(xi), grad(eta), grad(zeta)
    return J.reshape(-1), B.reshape(-1, 9).T


@pytest.mark.parametrize("case,tol", [(tanh_box, 2e-2), (rotated_cube, 1e-8), (conical_shell, 1e-3)])
def test_metrics_known_answer(oracle_lib, case, tol):
    shape, f = case()
    IM, JM, KM = shape
    k, j, i = _grid(IM, JM, KM)
    x, y, z = (np.asarray(v, dtype=float) for v in f(i, j, k))
    o = orc.OracleBlock(make_params(IM, JM, KM))
    o.calc_metrics(x, y, z)
    got = o.get_metrics()
    J, B = exact_metrics(shape, f)
    mse = [np.mean((got[m] - B[m]) ** 2) for m in range(9)] + [np.mean((got[9] - J) ** 2)]
    assert max(mse) <= tol, mse


def test_metric_ghosts_are_clamped(oracle_lib):
    """Ghost faces, edges and corners hold the nearest boundary node's metrics
    (src/metrics_kernel.cu:72-560)."""
    shape, f = conical_shell()
    IM, JM, KM = shape
    k, j, i = _grid(IM, JM, KM)
    x, y, z = (np.asarray(v, dtype=float) for v in f(i, j, k))
    o = orc.OracleBlock(make_params(IM, JM, KM))
    o.calc_metrics(x, y, z)
    g = o.get_metrics_ghosted().reshape(10, KM + 4, JM + 4, IM + 4)
    ci = np.clip(np.arange(-2, IM + 2), 0, IM - 1) + 2
    cj = np.clip(np.arange(-2, JM + 2), 0, JM - 1) + 2
    ck = np.clip(np.arange(-2, KM + 2), 0, KM - 1) + 2
    assert np.array_equal(g, g[:, ck][:, :, cj][:, :, :, ci])
