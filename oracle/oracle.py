"""ctypes wrapper of the CPU FP64 oracle (oracle/liborc.so).

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module, as the checker or the timed CPU baseline.
The oracle restates the reference's functions in the reference's own layout;
see cbns_oracle.cpp for the per-function citations.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liborc.so"
NG = 2
NEQ = 5

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    # local import keeps the oracle free of any dependency on the GPU library's loader
    from cbns3d_cuda_b200._abi import Params  # the struct layout only
    lib = C.CDLL(str(LIB))
    D = C.POINTER(C.c_double)
    V = C.c_void_p
    sig = {
        "orc_create": (V, [C.POINTER(Params)]),
        "orc_destroy": (None, [V]),
        "orc_calc_metrics": (None, [V, D, D, D]),
        "orc_get_metrics_ghosted": (None, [V, D]),
        "orc_get_metrics": (None, [V, D]),
        "orc_initial_condition": (None, [V]),
        "orc_calc_conservative": (None, [V, C.c_int]),
        "orc_set_conservative": (None, [V, D]),
        "orc_get_conservative": (None, [V, C.c_int, D]),
        "orc_get_primitive": (None, [V, D]),
        "orc_calc_primitive": (None, [V, C.c_int]),
        "orc_set_bc_calc_primitive": (None, [V, C.c_int]),
        "orc_calc_numerical_flux": (None, [V, C.c_int]),
        "orc_get_face_fluxes": (None, [V, D, D, D]),
        "orc_calc_viscous_terms": (None, [V]),
        "orc_calc_viscous_flux_contribution": (None, [V]),
        "orc_update_rk3": (None, [V, C.c_double, C.c_uint]),
        "orc_calc_dt": (C.c_double, [V]),
        "orc_solve": (C.c_int, [V, C.c_uint, C.c_double, D, C.POINTER(C.c_uint)]),
        "orc_eval_rhs": (None, [V, C.c_int, D]),
        "orc_calc_gradient": (None, [C.c_uint, C.c_uint, C.c_uint, D, D, D, D]),
        "orc_sensor_faces": (None, [V, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "orc_set_face_mask": (None, [V, C.c_void_p, C.c_long]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int | None):
    """OpenMP thread count for the oracle (must be set before the first parallel region)."""
    if n:
        os.environ["OMP_NUM_THREADS"] = str(n)


class OracleBlock:
    """Same operations as cbns3d_cuda_b200.Block, on the CPU in FP64."""

    def __init__(self, params):
        self.lib = load()
        self.p = params
        self.h = self.lib.orc_create(C.byref(params))
        if not self.h:
            raise ValueError("oracle: bad parameters")
        self.IM, self.JM, self.KM = params.IM, params.JM, params.KM
        self.IG, self.JG, self.KG = self.IM + 2 * NG, self.JM + 2 * NG, self.KM + 2 * NG

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def calc_metrics(self, x, y, z):
        a = [np.ascontiguousarray(v, dtype=np.float64).reshape(-1) for v in (x, y, z)]
        self.lib.orc_calc_metrics(self.h, *[_p(v) for v in a])

    def get_metrics(self):
        out = np.empty(10 * self.IM * self.JM * self.KM)
        self.lib.orc_get_metrics(self.h, _p(out))
        return out.reshape(10, -1)

    def get_metrics_ghosted(self):
        out = np.empty(10 * self.IG * self.JG * self.KG)
        self.lib.orc_get_metrics_ghosted(self.h, _p(out))
        return out.reshape(10, -1)

    def initial_condition(self):
        self.lib.orc_initial_condition(self.h)

    def calc_conservative(self, which=0):
        self.lib.orc_calc_conservative(self.h, which)

    def set_conservative(self, Q):
        q = np.ascontiguousarray(Q, dtype=np.float64).reshape(-1)
        self.lib.orc_set_conservative(self.h, _p(q))

    def get_conservative(self, which=0):
        q = np.empty(NEQ * self.IG * self.JG * self.KG)
        self.lib.orc_get_conservative(self.h, which, _p(q))
        return q

    def get_primitive(self):
        out = np.empty(7 * self.IG * self.JG * self.KG)
        self.lib.orc_get_primitive(self.h, _p(out))
        return out.reshape(7, -1)

    def calc_primitive(self, which=0):
        self.lib.orc_calc_primitive(self.h, which)

    def set_bc_calc_primitive(self, which=0):
        self.lib.orc_set_bc_calc_primitive(self.h, which)

    def calc_numerical_flux(self, which=0):
        self.lib.orc_calc_numerical_flux(self.h, which)

    def face_fluxes(self):
        IM, JM, KM = self.IM, self.JM, self.KM
        Ep = np.empty(NEQ * (IM - 1) * (JM - 2) * (KM - 2))
        Fp = np.empty(NEQ * (IM - 2) * (JM - 1) * (KM - 2))
        Gp = np.empty(NEQ * (IM - 2) * (JM - 2) * (KM - 1))
        self.lib.orc_get_face_fluxes(self.h, _p(Ep), _p(Fp), _p(Gp))
        return Ep, Fp, Gp

    def calc_viscous_terms(self):
        self.lib.orc_calc_viscous_terms(self.h)

    def calc_viscous_flux_contribution(self):
        self.lib.orc_calc_viscous_flux_contribution(self.h)

    def update_rk3(self, dt, stage):
        self.lib.orc_update_rk3(self.h, float(dt), int(stage))

    def calc_dt(self):
        return self.lib.orc_calc_dt(self.h)

    def solve(self, nsteps, t_end, t_cur=0.0):
        t = C.c_double(t_cur)
        n = C.c_uint()
        rc = self.lib.orc_solve(self.h, int(nsteps), float(t_end), C.byref(t), C.byref(n))
        return rc, t.value, n.value

    def eval_rhs(self, which=0):
        out = np.empty(NEQ * (self.IM - 2) * (self.JM - 2) * (self.KM - 2))
        self.lib.orc_eval_rhs(self.h, which, _p(out))
        return out

    def set_face_mask(self, mask=None):
        """Hybrid decisions (uint8 per face, 1 = WENO5) for later flux
        evaluations; None restores WENO5 everywhere."""
        if mask is None:
            self.lib.orc_set_face_mask(self.h, None, 0)
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        self.lib.orc_set_face_mask(self.h, m.ctypes.data, m.size)

    def sensor_faces(self, which=0):
        """(features n x 15, deviation n) of every face, i-, j-, then k-faces."""
        IM, JM, KM = self.IM, self.JM, self.KM
        n = (IM - 1) * (JM - 2) * (KM - 2) + (IM - 2) * (JM - 1) * (KM - 2) + (IM - 2) * (JM - 2) * (KM - 1)
        f = np.empty((n, 15), dtype=np.float32)
        d = np.empty(n, dtype=np.float32)
        self.lib.orc_sensor_faces(self.h, which, f.ctypes.data_as(C.POINTER(C.c_float)),
                                  d.ctypes.data_as(C.POINTER(C.c_float)))
        return f, d

    def init_like_reference(self, x, y, z, Q0=None):
        """calc_metrics, the start state and the first boundary pass of
        src/Block3d.cpp:217-233."""
        self.calc_metrics(x, y, z)
        if Q0 is None:
            self.initial_condition()
            self.calc_conservative(0)
        else:
            self.set_conservative(Q0)
            if self.p.viscous:
                self.calc_primitive(0)
        self.set_bc_calc_primitive(0)
        if self.p.viscous:
            self.calc_viscous_terms()


def calc_gradient(f):
    lib = load()
    KM, JM, IM = f.shape
    a = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
    out = [np.empty_like(a) for _ in range(3)]
    lib.orc_calc_gradient(IM, JM, KM, _p(a), *[_p(o) for o in out])
    return [o.reshape(f.shape) for o in out]
