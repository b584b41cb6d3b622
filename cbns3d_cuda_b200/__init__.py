"""B200 (sm_100a) implementation of the cbns3d_cuda RK3 right-hand-side path.

The compute path is the CUDA library ``libcbns_b200.so`` (C ABI in
include/cbns_b200.h).  ``Block`` is the Python mirror of the reference's host
API (namespace block3d_cuda): the same operations, in the same order, with the
same argument meaning; every call runs on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (BC_CHARACTERISTIC, BC_FARFIELD, BC_OGRID, BC_REFERENCE, DTV_FULL, DTV_REFERENCE, OGRID_WRAP,  # noqa: F401
                   CBNS_Q, CBNS_QP, PREC_FP64, PREC_HYBRID, PREC_SPLIT,
                   VISDIV_CENTERED, VISDIV_REFERENCE, CbnsError, Params)

__all__ = ["selftest_waits", "Block", "Batch", "Params", "CbnsError", "CBNS_Q", "CBNS_QP", "PREC_FP64", "PREC_SPLIT", "PREC_HYBRID",
           "VISDIV_REFERENCE", "VISDIV_CENTERED", "BC_REFERENCE", "BC_FARFIELD", "BC_CHARACTERISTIC", "BC_OGRID", "OGRID_WRAP",
           "DTV_REFERENCE", "DTV_FULL",
           "make_params"]

NG = 2
NEQ = 5


def make_params(IM, JM, KM, *, CFL=0.5, angle_attack=0.0, i_begin=1, i_end=0, Mach=0.5, Re=1.0e4, gamma=1.4,
                Pr=0.72, Pr_t=0.9, T_inf=288.15, viscous=False, precision=PREC_FP64,
                vis_divergence=VISDIV_REFERENCE, bc_mode=BC_REFERENCE, dt_viscous=DTV_REFERENCE) -> Params:
    p = Params()
    p.IM, p.JM, p.KM = IM, JM, KM
    p.CFL, p.angle_attack = CFL, angle_attack
    p.i_begin, p.i_end = i_begin, i_end
    p.Mach, p.Re, p.gamma, p.Pr, p.Pr_t, p.T_inf = Mach, Re, gamma, Pr, Pr_t, T_inf
    p.viscous, p.precision, p.vis_divergence = int(viscous), int(precision), int(vis_divergence)
    p.bc_mode = int(bc_mode)
    p.dt_viscous = int(dt_viscous)
    return p


class Block:
    """One curvilinear block on the GPU (the reference's Block3dData + block3d_cuda calls)."""

    def __init__(self, params: Params):
        self.lib = _abi.load()
        self.p = params
        h = C.c_void_p()
        _abi.check(self.lib.cbns_create(C.byref(params), C.byref(h)), "cbns_create")
        self.h = h
        self.IM, self.JM, self.KM = params.IM, params.JM, params.KM
        self.IG, self.JG, self.KG = self.IM + 2 * NG, self.JM + 2 * NG, self.KM + 2 * NG

    # lifecycle -------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            _abi.check(self.lib.cbns_destroy(self.h), "cbns_destroy")
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        """Wait for every call enqueued on the block's stream."""
        _abi.check(self.lib.cbns_synchronize(self.h), "cbns_synchronize")

    def set_stream(self, stream_ptr: int | None):
        _abi.check(self.lib.cbns_set_stream(self.h, C.c_void_p(stream_ptr or 0)), "cbns_set_stream")

    # setup and I/O ---------------------------------------------------------
    def calc_metrics(self, x: np.ndarray, y: np.ndarray, z: np.ndarray):
        a = [np.ascontiguousarray(v, dtype=np.float64).reshape(-1) for v in (x, y, z)]
        _abi.check(self.lib.cbns_calc_metrics(self.h, *[_abi.dptr(v) for v in a]), "cbns_calc_metrics")

    def get_metrics(self) -> np.ndarray:
        n = self.IM * self.JM * self.KM
        out = [np.empty(n) for _ in range(10)]
        _abi.check(self.lib.cbns_get_metrics(self.h, *[_abi.dptr(v) for v in out]), "cbns_get_metrics")
        return np.stack(out)

    def initial_condition(self):
        _abi.check(self.lib.cbns_initial_condition(self.h), "cbns_initial_condition")

    def calc_conservative(self, which=CBNS_Q):
        _abi.check(self.lib.cbns_calc_conservative(self.h, which), "cbns_calc_conservative")

    def set_conservative(self, Q: np.ndarray):
        q = np.ascontiguousarray(Q, dtype=np.float64).reshape(-1)
        assert q.size == NEQ * self.IG * self.JG * self.KG
        _abi.check(self.lib.cbns_set_conservative(self.h, _abi.dptr(q)), "cbns_set_conservative")

    def init_case(self, kind: int, x, y, z, prm):
        """The case's initial state formed on the device (cbns_init_case):
        kind _abi.CASE_*, prm its parameters, x/y/z the grid (KM, JM, IM)."""
        a = [np.ascontiguousarray(v, dtype=np.float64).reshape(-1) for v in (x, y, z)]
        pv = np.ascontiguousarray(prm, dtype=np.float64).reshape(-1)
        _abi.check(self.lib.cbns_init_case(self.h, int(kind), *(_abi.dptr(v) for v in a), _abi.dptr(pv), len(pv)),
                   "cbns_init_case")

    def get_conservative(self, which=CBNS_Q, out: np.ndarray | None = None) -> np.ndarray:
        n = NEQ * self.IG * self.JG * self.KG
        q = out if out is not None else np.empty(n)
        _abi.check(self.lib.cbns_get_conservative(self.h, which, _abi.dptr(q)), "cbns_get_conservative")
        return q

    def get_primitive(self) -> np.ndarray:
        n = self.IG * self.JG * self.KG
        out = [np.empty(n) for _ in range(6)]
        _abi.check(self.lib.cbns_get_primitive(self.h, *[_abi.dptr(v) for v in out]), "cbns_get_primitive")
        return np.stack(out)

    # the RK3 right-hand-side path -----------------------------------------
    def set_bc_calc_primitive(self, which=CBNS_Q):
        _abi.check(self.lib.cbns_set_bc_calc_primitive(self.h, which), "cbns_set_bc_calc_primitive")

    def calc_primitive(self, which=CBNS_Q):
        _abi.check(self.lib.cbns_calc_primitive(self.h, which), "cbns_calc_primitive")

    def calc_numerical_flux(self, which=CBNS_Q):
        _abi.check(self.lib.cbns_calc_numerical_flux(self.h, which), "cbns_calc_numerical_flux")

    def calc_viscous_terms(self):
        _abi.check(self.lib.cbns_calc_viscous_terms(self.h), "cbns_calc_viscous_terms")

    def calc_viscous_flux_contribution(self):
        _abi.check(self.lib.cbns_calc_viscous_flux_contribution(self.h), "cbns_calc_viscous_flux_contribution")

    def update_rk3(self, dt: float, stage: int):
        _abi.check(self.lib.cbns_update_rk3(self.h, float(dt), int(stage)), "cbns_update_rk3")

    def calc_dt(self) -> float:
        dt = C.c_double()
        _abi.check(self.lib.cbns_calc_dt(self.h, C.byref(dt)), "cbns_calc_dt")
        return dt.value

    def eval_rhs(self, which=CBNS_Q) -> np.ndarray:
        out = np.empty(NEQ * (self.IM - 2) * (self.JM - 2) * (self.KM - 2))
        _abi.check(self.lib.cbns_eval_rhs(self.h, which, _abi.dptr(out)), "cbns_eval_rhs")
        return out

    # whole steps ------------------------------------------------------------
    def set_time(self, t: float):
        _abi.check(self.lib.cbns_set_time(self.h, float(t)), "cbns_set_time")

    def get_time(self) -> tuple[float, float]:
        t, dt = C.c_double(), C.c_double()
        _abi.check(self.lib.cbns_get_time(self.h, C.byref(t), C.byref(dt)), "cbns_get_time")
        return t.value, dt.value

    def run(self, nsteps: int, t_end: float = 1.0e30) -> int:
        done = C.c_uint()
        _abi.check(self.lib.cbns_run(self.h, int(nsteps), float(t_end), C.byref(done)), "cbns_run")
        return done.value

    def run_async(self, nsteps: int, t_end: float = 1.0e30):
        _abi.check(self.lib.cbns_run_async(self.h, int(nsteps), float(t_end)), "cbns_run_async")

    def step_like_reference(self, t_cur: float, t_end: float) -> float:
        """One step of the time loop of src/Block3d.cpp:239-287 through the
        per-call entry points; returns the new t_cur."""
        dt = self.calc_dt()
        if t_end - t_cur < dt:
            dt = t_end - t_cur
        t_cur += dt
        visc = bool(self.p.viscous)
        for s in (1, 2, 3):
            self.calc_numerical_flux(CBNS_Q if s == 1 else CBNS_QP)
            if visc:
                self.calc_viscous_flux_contribution()
            self.update_rk3(dt, s)
            self.set_bc_calc_primitive(CBNS_Q if s == 3 else CBNS_QP)
            if visc:
                self.calc_viscous_terms()
        return t_cur

    # hybrid flux (precision PREC_HYBRID) -------------------------------------
    def sensor_load(self, params: np.ndarray, tau: float):
        """Install the sensor network (CBNS_SENSOR_NPARAM floats) and its threshold."""
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        if p.size != 1601:
            raise ValueError(f"sensor parameters: expected 1601 values, got {p.size}")
        _abi.check(self.lib.cbns_sensor_load(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), float(tau)),
                   "cbns_sensor_load")

    def sensor_audit(self, stride: int = 97, bound: float = 1.0e-2):
        _abi.check(self.lib.cbns_sensor_audit(self.h, int(stride), float(bound)), "cbns_sensor_audit")

    def sensor_interval(self, every: int = 3):
        _abi.check(self.lib.cbns_sensor_interval(self.h, int(every)), "cbns_sensor_interval")

    def sensor_stats(self) -> dict:
        s = _abi.SensorStats()
        _abi.check(self.lib.cbns_sensor_stats_get(self.h, C.byref(s)), "cbns_sensor_stats_get")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def sensor_mask(self) -> tuple[np.ndarray, bool]:
        """(decisions of the latest sensor evaluation, 1 = WENO5; audit forced WENO5)."""
        n = self.sensor_stats()["faces_per_step"]
        m = np.empty(n, dtype=np.uint8)
        f = C.c_int()
        _abi.check(self.lib.cbns_sensor_mask_get(self.h, m.ctypes.data, n, C.byref(f)), "cbns_sensor_mask_get")
        return m, bool(f.value)

    def sensor_stats_reset(self):
        _abi.check(self.lib.cbns_sensor_stats_reset(self.h), "cbns_sensor_stats_reset")

    def autotune(self) -> int:
        v = C.c_int()
        _abi.check(self.lib.cbns_autotune(self.h, C.byref(v)), "cbns_autotune")
        return v.value

    def stage_variant(self, variant: int = -1) -> int:
        """Select compiled stage-kernel variant `variant` (-1: only query);
        returns the number of variants."""
        n = C.c_int()
        _abi.check(self.lib.cbns_stage_variant(self.h, int(variant), C.byref(n)), "cbns_stage_variant")
        return n.value

    def stage_kchunk(self, kchunk: int = -1) -> int:
        """Use k chunks of `kchunk` planes in the stage kernel (-1: only
        query); returns the chunk in use."""
        n = C.c_int()
        _abi.check(self.lib.cbns_stage_kchunk(self.h, int(kchunk), C.byref(n)), "cbns_stage_kchunk")
        return n.value

    # timing -----------------------------------------------------------------
    def prof_enable(self, on=True):
        _abi.check(self.lib.cbns_prof_enable(self.h, int(on)), "cbns_prof_enable")

    def prof_reset(self):
        _abi.check(self.lib.cbns_prof_reset(self.h), "cbns_prof_reset")

    def prof_read(self, kernel_id: int) -> tuple[float, int]:
        ms, n = C.c_double(), C.c_uint()
        _abi.check(self.lib.cbns_prof_read(self.h, kernel_id, C.byref(ms), C.byref(n)), "cbns_prof_read")
        return ms.value, n.value

    def launch_count(self) -> int:
        n = C.c_ulonglong()
        _abi.check(self.lib.cbns_launch_count(self.h, C.byref(n)), "cbns_launch_count")
        return n.value


class Batch:
    """Independent blocks advanced together (cbns_batch_*): one persistent
    work-queue launch of the stage kernel per RK stage for all blocks, per-block
    dt, a whole step as one CUDA graph.  The blocks stay usable on their own
    (get_conservative, ...); close the batch before them."""

    def __init__(self, blocks, stream_ptr: int | None = None):
        self.lib = _abi.load()
        self.blocks = list(blocks)
        arr = (C.c_void_p * len(self.blocks))(*[b.h.value if isinstance(b.h, C.c_void_p) else b.h
                                                 for b in self.blocks])
        h = C.c_void_p()
        _abi.check(self.lib.cbns_batch_create(arr, len(self.blocks), C.c_void_p(stream_ptr or 0), C.byref(h)),
                   "cbns_batch_create")
        self.h = h

    def run(self, nsteps: int, t_end: float = 1.0e30) -> int:
        n = C.c_uint()
        _abi.check(self.lib.cbns_batch_run(self.h, int(nsteps), float(t_end), C.byref(n)), "cbns_batch_run")
        return n.value

    def run_async(self, nsteps: int, t_end: float = 1.0e30):
        _abi.check(self.lib.cbns_batch_run_async(self.h, int(nsteps), float(t_end)), "cbns_batch_run_async")

    def close(self):
        if getattr(self, "h", None):
            _abi.check(self.lib.cbns_batch_destroy(self.h), "cbns_batch_destroy")
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def calc_gradient(f: np.ndarray):
    """4th-order gradient of a (KM, JM, IM) field on the GPU (src/calc_gradient.cu)."""
    lib = _abi.load()
    KM, JM, IM = f.shape
    a = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
    out = [np.empty_like(a) for _ in range(3)]
    _abi.check(lib.cbns_calc_gradient(IM, JM, KM, _abi.dptr(a), *[_abi.dptr(o) for o in out]), "cbns_calc_gradient")
    return [o.reshape(f.shape) for o in out]


def selftest_waits() -> dict:
    """Run the bounded waits' time-out path on the GPU (cbns_selftest_waits):
    whether the tensor-core MMA wait and the TMA transaction wait each reported
    a time-out on a barrier nothing completes, and how long each took."""
    lib = _abi.load()
    a, b = C.c_int(-1), C.c_int(-1)
    sa, sb = C.c_double(), C.c_double()
    _abi.check(lib.cbns_selftest_waits(C.byref(a), C.byref(b), C.byref(sa), C.byref(sb)), "cbns_selftest_waits")
    return {"mma_timed_out": a.value, "tma_timed_out": b.value, "mma_seconds": sa.value, "tma_seconds": sb.value}
