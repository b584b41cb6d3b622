"""ctypes binding of libcbns_b200.so (include/cbns_b200.h).

The shared library is built in-tree by ``cbns3d_cuda_b200.build``; loading
fails loudly when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcbns_b200.so"

CBNS_OK = 0
CBNS_ERR_ARG = 1
CBNS_ERR_CUDA = 2
CBNS_ERR_NAN_DT = 3
CBNS_ERR_STATE = 4
CBNS_ERR_UNSUPPORTED = 5
CBNS_ERR_NOMEM = 6
CBNS_ERR_TOO_LARGE = 7

CBNS_Q = 0
CBNS_QP = 1

PREC_FP64 = 0
PREC_SPLIT = 1
PREC_HYBRID = 2

VISDIV_REFERENCE = 0
VISDIV_CENTERED = 1

CASE_VORTEX = 0
CASE_BLAST = 1
CASE_SHOCK_VORTEX = 2

BC_REFERENCE = 0  # the reference's boundary conditions (parity contract)
BC_FARFIELD = 1   # every boundary and ghost node holds the state it was set to
BC_CHARACTERISTIC = 2  # Riemann-invariant far field against the free stream on every face
BC_OGRID = 3      # i wraps around (OGRID_WRAP copied points either side), wall j = 0, characteristic j = JM-1
OGRID_WRAP = 4
DTV_REFERENCE = 0  # viscous dt term scaled by the local |u|/c, as the reference
DTV_FULL = 1       # viscous dt term without that factor (wall-resolved grids)


class Params(C.Structure):
    """cbns_params: the fields Block3d::read_input fills plus run-time switches."""

    _fields_ = [
        ("IM", C.c_uint), ("JM", C.c_uint), ("KM", C.c_uint),
        ("CFL", C.c_double), ("angle_attack", C.c_double),
        ("i_begin", C.c_uint), ("i_end", C.c_uint),
        ("Mach", C.c_double), ("Re", C.c_double), ("gamma", C.c_double),
        ("Pr", C.c_double), ("Pr_t", C.c_double), ("T_inf", C.c_double),
        ("viscous", C.c_int), ("precision", C.c_int), ("vis_divergence", C.c_int),
        ("bc_mode", C.c_int), ("dt_viscous", C.c_int), ("reserved", C.c_int * 3),
    ]


class SensorStats(C.Structure):
    """cbns_sensor_stats: counters of the hybrid flux's sensor and audit."""

    _fields_ = [
        ("weno_faces", C.c_ulonglong), ("audit_faces", C.c_ulonglong),
        ("audit_fail_steps", C.c_uint), ("audit_max", C.c_float),
        ("sensor_fail", C.c_int), ("faces_per_step", C.c_ulonglong),
    ]


# (name, restype, argtypes) of every exported entry point
_D = C.POINTER(C.c_double)
_V = C.c_void_p
SIGNATURES = [
    ("cbns_create", C.c_int, [C.POINTER(Params), C.POINTER(_V)]),
    ("cbns_destroy", C.c_int, [_V]),
    ("cbns_set_stream", C.c_int, [_V, _V]),
    ("cbns_status_string", C.c_char_p, [C.c_int]),
    ("cbns_calc_metrics", C.c_int, [_V, _D, _D, _D]),
    ("cbns_get_metrics", C.c_int, [_V] + [_D] * 10),
    ("cbns_initial_condition", C.c_int, [_V]),
    ("cbns_calc_conservative", C.c_int, [_V, C.c_int]),
    ("cbns_set_conservative", C.c_int, [_V, _D]),
    ("cbns_init_case", C.c_int, [_V, C.c_int, _D, _D, _D, _D, C.c_uint]),
    ("cbns_get_conservative", C.c_int, [_V, C.c_int, _D]),
    ("cbns_get_primitive", C.c_int, [_V, _D, _D, _D, _D, _D, _D]),
    ("cbns_set_bc_calc_primitive", C.c_int, [_V, C.c_int]),
    ("cbns_calc_primitive", C.c_int, [_V, C.c_int]),
    ("cbns_calc_numerical_flux", C.c_int, [_V, C.c_int]),
    ("cbns_calc_viscous_terms", C.c_int, [_V]),
    ("cbns_calc_viscous_flux_contribution", C.c_int, [_V]),
    ("cbns_update_rk3", C.c_int, [_V, C.c_double, C.c_uint]),
    ("cbns_calc_dt", C.c_int, [_V, _D]),
    ("cbns_run", C.c_int, [_V, C.c_uint, C.c_double, C.POINTER(C.c_uint)]),
    ("cbns_run_async", C.c_int, [_V, C.c_uint, C.c_double]),
    ("cbns_set_time", C.c_int, [_V, C.c_double]),
    ("cbns_get_time", C.c_int, [_V, _D, _D]),
    ("cbns_eval_rhs", C.c_int, [_V, C.c_int, _D]),
    ("cbns_calc_gradient", C.c_int, [C.c_uint, C.c_uint, C.c_uint, _D, _D, _D, _D]),
    ("cbns_autotune", C.c_int, [_V, C.POINTER(C.c_int)]),
    ("cbns_stage_variant", C.c_int, [_V, C.c_int, C.POINTER(C.c_int)]),
    ("cbns_stage_kchunk", C.c_int, [_V, C.c_int, C.POINTER(C.c_int)]),
    ("cbns_selftest_waits", C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]),
    ("cbns_synchronize", C.c_int, [_V]),
    ("cbns_sensor_sample", C.c_int,
     [_V, C.c_int, C.c_uint, C.c_uint, _V, _V, _V, _V, C.c_uint, C.POINTER(C.c_uint)]),
    ("cbns_mlp_grad", C.c_int, [_V, _V, _V, C.c_uint, C.c_float, _V, _V, _V]),
    ("cbns_mlp_adam", C.c_int, [_V, _V, _V, _V, C.c_uint, C.c_float, _V]),
    ("cbns_mlp_predict", C.c_int, [_V, _V, C.c_uint, _V, C.c_int, _V, _V]),
    ("cbns_sensor_load", C.c_int, [_V, C.POINTER(C.c_float), C.c_float]),
    ("cbns_sensor_load_file", C.c_int, [_V, C.c_char_p]),
    ("cbns_batch_create", C.c_int, [C.POINTER(_V), C.c_uint, _V, C.POINTER(_V)]),
    ("cbns_batch_destroy", C.c_int, [_V]),
    ("cbns_batch_run", C.c_int, [_V, C.c_uint, C.c_double, C.POINTER(C.c_uint)]),
    ("cbns_batch_run_async", C.c_int, [_V, C.c_uint, C.c_double]),
    ("cbns_sensor_audit", C.c_int, [_V, C.c_uint, C.c_float]),
    ("cbns_sensor_interval", C.c_int, [_V, C.c_uint]),
    ("cbns_sensor_stats_get", C.c_int, [_V, C.POINTER(SensorStats)]),
    ("cbns_sensor_stats_reset", C.c_int, [_V]),
    ("cbns_sensor_mask_get", C.c_int, [_V, _V, C.c_ulonglong, C.POINTER(C.c_int)]),
    ("cbns_prof_enable", C.c_int, [_V, C.c_int]),
    ("cbns_prof_read", C.c_int, [_V, C.c_int, _D, C.POINTER(C.c_uint)]),
    ("cbns_prof_reset", C.c_int, [_V]),
    ("cbns_launch_count", C.c_int, [_V, C.POINTER(C.c_ulonglong)]),
]

_lib = None


def load(path: Path | str | None = None):
    """Load the library (once).  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m cbns3d_cuda_b200.build`")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class CbnsError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = load().cbns_status_string(code).decode()
        super().__init__(f"{where}: {msg} (status {code})")
        self.code = code


def check(code: int, where: str) -> None:
    if code != CBNS_OK:
        raise CbnsError(code, where)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)
