"""cbns_calc_gradient_noalloc, the gradient entry point for callers that cannot
allocate device memory (hosts whose device memory belongs to their own pool
allocator or a fixed budget, or paths where cudaMalloc's device-wide
synchronisation is not acceptable).  It must give what the allocating
cbns_calc_gradient gives, on consecutive calls that reuse its one fixed
device array, leave the device's free memory unchanged, and refuse sizes
above CBNS_NOALLOC_MAX_POINTS.

Collected last on purpose: a run that stops at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from cbns3d_cuda_b200 import _abi

pytestmark = pytest.mark.gpu

MAX_POINTS = 262144  # CBNS_NOALLOC_MAX_POINTS in include/cbns_b200.h
_D = C.POINTER(C.c_double)


def _lib():
    lib = _abi.load()
    for name in ("cbns_calc_gradient_noalloc", "cbns_calc_gradient"):
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = [C.c_uint, C.c_uint, C.c_uint, _D, _D, _D, _D]
    return lib


def _grad(fn, f):
    KM, JM, IM = f.shape
    out = [np.empty_like(f) for _ in range(3)]
    rc = fn(IM, JM, KM, *[_abi.dptr(a) for a in [f] + out])
    return rc, out


def test_noalloc_gradient_matches_allocating_entry_point_on_consecutive_calls():
    lib = _lib()
    rng = np.random.default_rng(11)
    # two calls in a row on the shared array: a small field, then one of exactly
    # the maximum size (which overwrites everything the first call left there)
    for shape in [(20, 30, 40), (64, 64, 64)]:
        k, j, i = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
        f = np.ascontiguousarray(np.sin(0.3 * i) * np.cos(0.2 * j) + 0.01 * k * k + rng.standard_normal(shape))
        rc_ref, ref = _grad(lib.cbns_calc_gradient, f)
        rc, got = _grad(lib.cbns_calc_gradient_noalloc, f)
        assert rc_ref == _abi.CBNS_OK and rc == _abi.CBNS_OK
        for a, b in zip(got, ref):
            scale = np.max(np.abs(b))
            assert np.max(np.abs(a - b)) <= 1e-12 * scale


def test_noalloc_gradient_allocates_nothing():
    """Free device memory is the same before and after warmed-up calls."""
    import torch

    lib = _lib()
    f = np.ascontiguousarray(np.random.default_rng(3).standard_normal((32, 48, 40)))
    rc, _ = _grad(lib.cbns_calc_gradient_noalloc, f)  # warm-up: address lookup, module load
    assert rc == _abi.CBNS_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        rc, _ = _grad(lib.cbns_calc_gradient_noalloc, f)
        assert rc == _abi.CBNS_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_gradient_rejects_oversize_request():
    lib = _lib()
    f = np.zeros((64, 64, 65))
    assert f.size > MAX_POINTS
    rc, _ = _grad(lib.cbns_calc_gradient_noalloc, f)
    assert rc == _abi.CBNS_ERR_TOO_LARGE
