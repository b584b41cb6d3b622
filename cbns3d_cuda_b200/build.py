"""Build the B200 library and driver in-tree with nvcc (sm_100a).

Outputs
  cbns3d_cuda_b200/libcbns_b200.so   C ABI (include/cbns_b200.h) + block3d_cuda shims
  cbns3d_cuda_b200/bin/cbns3d_b200   host driver (reads input.txt like the reference)

Usage: python -m cbns3d_cuda_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
BUILD = ROOT / "_build" / "cbns"
LIB = PKG / "libcbns_b200.so"
EXE = PKG / "bin" / "cbns3d_b200"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I" + str(ROOT / "include")]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx() -> str:
    # the environment's CXX may lack system headers/libs; prefer the system g++
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    nvcc = _nvcc()
    jobs = []
    objs = []
    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + headers):
            cmd = [nvcc] + NVFLAGS + ["-ccbin", _host_cxx(), "-c", str(s), "-o", str(o)]
            jobs.append(cmd)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or not LIB.exists():
        _run([nvcc] + ARCH + ["-ccbin", _host_cxx(), "-shared", "-cudart", "static", "-o", str(LIB)] +
             [str(o) for o in objs])
    host_srcs = sorted(HOST.glob("*.cpp"))
    if force or not _newer(EXE, host_srcs + list(HOST.glob("*.h")) + [LIB]):
        _run([nvcc, "-ccbin", _host_cxx(), "-cudart", "none", "-O2", "-std=c++17", "-I" + str(ROOT / "include"),
              "-o", str(EXE)] + [str(s) for s in host_srcs] +
             ["-L" + str(PKG), "-lcbns_b200", "-Xlinker", "-rpath=$ORIGIN/.."])
    if verbose:
        print(f"built {LIB} and {EXE}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
