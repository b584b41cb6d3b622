"""Comparison helpers shared by the tests."""
import numpy as np


def rel_linf(a, b):
    """max |a - b| / max |b| (the parity measure of every FP64 comparison)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def per_var_rel_linf(Qa, Qb):
    """relative L-infinity per conservative variable (last axis of size 5)."""
    Qa = np.asarray(Qa).reshape(-1, 5)
    Qb = np.asarray(Qb).reshape(-1, 5)
    return [rel_linf(Qa[:, n], Qb[:, n]) for n in range(5)]


def interior(Q, shape, ng=2):
    """(KG,JG,IG,5) view restricted to the IM x JM x KM grid nodes."""
    IM, JM, KM = shape
    q = np.asarray(Q).reshape(KM + 2 * ng, JM + 2 * ng, IM + 2 * ng, -1)
    return q[ng:ng + KM, ng:ng + JM, ng:ng + IM]
