"""The C-ABI library loads without a GPU and exports every declared symbol."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "cbns3d_cuda_b200" / "libcbns_b200.so"


@pytest.fixture(scope="module")
def built():
    if not LIB.exists():
        from cbns3d_cuda_b200 import build
        build.build()
    return LIB


def declared_c_symbols():
    text = (ROOT / "include" / "cbns_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|int)\s+(cbns_\w+)\s*\(", text, re.M)))


def declared_shim_functions():
    text = (ROOT / "include" / "block3d_cuda.h").read_text()
    body = text[text.index("namespace block3d_cuda"):]
    return sorted(set(re.findall(r"^\s*(?:void|value_type)\s+(\w+)\s*\(", body, re.M)))


def test_c_abi_symbols_exported(built):
    out = subprocess.run(["nm", "-D", "--defined-only", str(built)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (\w+)$", out, re.M))
    decl = declared_c_symbols()
    assert len(decl) >= 25
    missing = [s for s in decl if s not in exported]
    assert not missing, missing


def test_block3d_cuda_shims_exported(built):
    out = subprocess.run(["nm", "-DC", "--defined-only", str(built)], capture_output=True, text=True,
                         check=True).stdout
    decl = declared_shim_functions()
    assert {"calc_numerical_flux", "update_rk3", "set_bc_calc_primitive", "calc_dt",
            "calc_viscous_terms", "calc_viscous_flux_contribution", "calc_primitive"} <= set(decl)
    missing = [f for f in decl if f"block3d_cuda::{f}(" not in out]
    assert not missing, missing


def test_library_loads_and_binds(built):
    from cbns3d_cuda_b200 import _abi
    lib = _abi.load()
    for name, _, _ in _abi.SIGNATURES:
        assert hasattr(lib, name)
    assert lib.cbns_status_string(_abi.CBNS_ERR_NAN_DT).decode().startswith("An error occurred")


def test_bad_params_rejected_without_gpu(built):
    """Argument checks run before any CUDA call."""
    import ctypes as C
    from cbns3d_cuda_b200 import _abi, make_params
    lib = _abi.load()
    h = C.c_void_p()
    p = make_params(3, 10, 10)
    assert lib.cbns_create(C.byref(p), C.byref(h)) == _abi.CBNS_ERR_ARG
    p = make_params(10, 10, 10, precision=7)
    assert lib.cbns_create(C.byref(p), C.byref(h)) == _abi.CBNS_ERR_ARG
    assert lib.cbns_create(None, C.byref(h)) == _abi.CBNS_ERR_ARG


def test_bad_boundary_modes_rejected_without_gpu(built):
    import ctypes as C
    from cbns3d_cuda_b200 import _abi, make_params
    lib = _abi.load()
    h = C.c_void_p()
    p = make_params(20, 10, 10, bc_mode=4)
    assert lib.cbns_create(C.byref(p), C.byref(h)) == _abi.CBNS_ERR_ARG
    p = make_params(2 * _abi.OGRID_WRAP + 5, 10, 10, bc_mode=_abi.BC_OGRID)  # periodic line of 5 < 6 points
    assert lib.cbns_create(C.byref(p), C.byref(h)) == _abi.CBNS_ERR_ARG


def test_header_constants_match_the_binding():
    import re
    from pathlib import Path
    from cbns3d_cuda_b200 import _abi
    hdr = (Path(__file__).resolve().parents[1] / "include" / "cbns_b200.h").read_text()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+CBNS_(\w+)\s+(-?\d+)\b", hdr)}
    for name in ("BC_REFERENCE", "BC_FARFIELD", "BC_CHARACTERISTIC", "BC_OGRID", "OGRID_WRAP", "PREC_FP64",
                 "PREC_SPLIT", "PREC_HYBRID", "VISDIV_REFERENCE", "VISDIV_CENTERED", "ERR_ARG", "ERR_NAN_DT"):
        py = getattr(_abi, name, None)
        if py is None:
            py = getattr(_abi, "CBNS_" + name)
        assert defs[name] == py, name
