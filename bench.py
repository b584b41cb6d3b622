#!/usr/bin/env python
"""Throughput of the RK3 right-hand-side path: cell-updates per second.

One step = one full SSP-RK3 step (three fused stage kernels, boundary
conditions, device-side CFL dt) of one block of synthetic input.  Default
workload: the shock-vortex case of 256 x 256 x 128 nodes (inviscid; inputs
larger than L2, so no flush is needed).  A cell-update is one interior node
advanced one step; N_upd = (IM-2)(JM-2)(KM-2).

  value   device-resident throughput of the split-precision path (FP32 flux
          arithmetic, FP64 state/metrics/reductions), timed with CUDA events on
          the launch stream; its density L2 error against the FP64 path after
          the same steps is reported and must stay <= 1e-5.
  paths   the same for the plain FP64 path (parity with the reference).
  e2e     the reference-style host-driven solve through the C ABI
          (block3d_cuda call sequence: dt read back every step, dt passed per
          stage), with the state uploaded from pinned host memory before and
          downloaded after the K steps inside the timed region.
  roofline  HBM roofline of the dominant kernel (the fused stage kernel).
  cpu_baseline  the FP64 CPU oracle (OpenMP, all host cores) on a bounded sample.

--impl reference runs the reference's own build (oracle/_ref, compiled from its
sources) on the same case through its own executable and times it from its
"Elapsed Time" output (difference of a W-step and a (W+K)-step run).

Multi-GPU: the path is one block on one GPU, so --gpus N runs N independent
replicas (weak scaling); value is the sum over ranks, time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# bytes per cell-update the kernel must move: per stage the stage input (40 B),
# the metrics (80 B) and the output (40 B), plus the RK base in stages 2 and 3
ALG_BYTES_PER_UPDATE = 560.0


def args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="shock_vortex", choices=["shock_vortex", "blast", "vortex"])
    ap.add_argument("--size", default=None, help="IMxJMxKM (default: the case's config size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def make_case(name, size):
    from cbns3d_cuda_b200 import cases
    if name == "shock_vortex":
        IM, JM, KM = size or (256, 256, 128)
        return cases.case_shock_vortex(IM, JM, KM), f"shock-vortex {IM}x{JM}x{KM} (configs[3] grid), inviscid"
    if name == "blast":
        IM, JM, KM = size or (384, 384, 384)
        return cases.case_blast(IM, JM, KM), f"spherical blast {IM}x{JM}x{KM} (configs[2]), inviscid"
    IM, JM, KM = size or (64, 32, 16)
    return cases.case_vortex(IM, JM, KM), f"isentropic vortex {IM}x{JM}x{KM} (configs[0]), inviscid"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = gpu_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            self.p.wait(timeout=10)

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if len(r) > 8]
        mx = [float(r[2]) for r in rows if len(r) > 8]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) > 8:
                for n, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def init_block(case, precision):
    from cbns3d_cuda_b200 import CBNS_Q, Block, make_params
    p = dict(case.params)
    p["precision"] = precision
    b = Block(make_params(*case.shape, **p))
    b.calc_metrics(case.x, case.y, case.z)
    b.set_conservative(case.Q0)
    b.set_bc_calc_primitive(CBNS_Q)
    return b


def n_updates(case):
    IM, JM, KM = case.shape
    return (IM - 2) * (JM - 2) * (KM - 2)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def device_pass(case, precision, K, W, torch, dist):
    """W untimed steps, then K timed steps with per-kernel events; returns
    (ms, block, per-kernel stats, launches)."""
    b = init_block(case, precision)
    stream = torch.cuda.Stream()  # a real stream: the legacy default stream cannot be graph-captured
    b.set_stream(stream.cuda_stream)
    b.torch_stream = stream
    b.variant = b.autotune()
    b.set_time(0.0)
    b.run(W)
    b.prof_enable(True)
    b.prof_reset()
    l0 = b.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run_async(K)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = b.launch_count() - l0
    kern = {kid: b.prof_read(kid) for kid in range(4)}
    b.prof_enable(False)
    return ms, b, kern, launches


def graph_pass(b, K, torch):
    """The same steps replayed from the CUDA graph (no per-kernel events)."""
    stream = b.torch_stream
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run_async(K)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def e2e_pass(case, K, torch):
    """Host-driven solve through the C ABI with host buffers (pinned)."""
    from cbns3d_cuda_b200 import CBNS_Q, PREC_SPLIT, _abi
    b = init_block(case, PREC_SPLIT)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    n = case.Q0.size
    hin = torch.empty(n, dtype=torch.float64, pin_memory=True)
    hout = torch.empty(n, dtype=torch.float64, pin_memory=True)
    hin.numpy()[:] = case.Q0.reshape(-1)
    # warm-up (first-call costs) outside the timed region
    t = b.step_like_reference(0.0, 1e30)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _abi.check(b.lib.cbns_set_conservative(b.h, _abi.dptr(hin.numpy())), "set_conservative")
    b.set_bc_calc_primitive(CBNS_Q)
    t = 0.0
    for _ in range(K):
        t = b.step_like_reference(t, 1e30)
    _abi.check(b.lib.cbns_get_conservative(b.h, CBNS_Q, _abi.dptr(hout.numpy())), "get_conservative")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    assert np.isfinite(hout.numpy()).all()
    state_bytes = n * 8
    b.close()
    return ms, {"h2d_bytes_per_step": state_bytes / K + 3 * 8, "d2h_bytes_per_step": state_bytes / K + 8}


def cpu_baseline(case, budget_s=15.0):
    from cbns3d_cuda_b200 import make_params
    from oracle import oracle as orc
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    o = orc.OracleBlock(make_params(*case.shape, **case.params))
    o.init_like_reference(case.x, case.y, case.z, case.Q0)
    steps, t0 = 0, time.perf_counter()
    t = 0.0
    while True:
        rc, t, n = o.solve(1, 1e30, t)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= 3:
            break
    o.close()
    return {"value": n_updates(case) * steps / el, "unit": "cell-updates/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port", "sample": f"{steps} RK3 step(s) of the same {case.shape} case, FP64 oracle "
                                      f"(C++/OpenMP restatement of the reference kernels), {el:.1f} s"}


def run_ours(a):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    else:
        torch.cuda.set_device(0)
    from cbns3d_cuda_b200 import PREC_FP64, PREC_SPLIT
    size = tuple(int(v) for v in a.size.split("x")) if a.size else None
    case, wl = make_case(a.case, size)
    K, W = a.steps, a.warmup
    N = n_updates(case)

    # plain FP64 path
    ms64, b64, kern64, _ = device_pass(case, PREC_FP64, K, W, torch, dist)
    q64 = b64.get_conservative()
    # split-precision path (headline), clocks sampled during its timed region
    with Clocks(local) as clk:
        ms32, b32, kern32, launches = device_pass(case, PREC_SPLIT, K, W, torch, dist)
    clocks = clk.summary()
    q32 = b32.get_conservative()
    variant32 = b32.variant
    IM, JM, KM = case.shape
    r64 = q64.reshape(KM + 4, JM + 4, IM + 4, 5)[2:-2, 2:-2, 2:-2, 0]
    r32 = q32.reshape(KM + 4, JM + 4, IM + 4, 5)[2:-2, 2:-2, 2:-2, 0]
    rho_l2 = float(np.sqrt(np.mean((r32 - r64) ** 2) / np.mean(r64 ** 2)))
    rho_linf = float(np.max(np.abs(r32 - r64)) / np.max(np.abs(r64)))
    gms32 = graph_pass(b32, K, torch)
    b64.close()
    b32.close()

    def reduce_max(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms32, ms64, gms32 = reduce_max(ms32), reduce_max(ms64), reduce_max(gms32)
    value = world * N * K / (ms32 / 1e3)
    value64 = world * N * K / (ms64 / 1e3)

    e2e = None
    if not a.no_e2e:
        ems, eb = e2e_pass(case, K, torch)
        ems = reduce_max(ems)
        e2e = {"value": world * N * K / (ems / 1e3), "unit": "cell-updates/s", **eb}

    peak, peak_kind = measured_peaks()
    st_ms, st_n = kern32[0]
    alg_per_launch = ALG_BYTES_PER_UPDATE / 3.0 * N
    achieved = alg_per_launch / (st_ms / st_n / 1e3) / 1e9 if st_n else None
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        t = json.loads(tf.read_text())
        if "stage_bytes_per_update" in t:
            traffic = t["stage_bytes_per_update"] / 3.0 * N
    st64_ms, st64_n = kern64[0]
    if rank == 0:
        cpu = None if a.no_cpu_baseline else cpu_baseline(case)
        line = {
            "metric": "cell-updates/s: learned-hybrid FP32 vs plain FP64 WENO5, same B200, rho-L2<=1e-5",
            "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms32 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 flux / f64 state", "data": "synthetic",
            "config": {"workload": wl, "path": "split precision (FP32 WENO5-char/LF flux, FP64 state, metrics, dt)",
                       "grid": list(case.shape), "cell_updates_per_step": N, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (3 state buffers + 10 metric arrays)",
                       "learned_sensor": "not built: value is the split path without the sensor"},
            "paths": {"fp64": {"value": value64, "ms_per_step": ms64 / K, "stage_kernel_ms": st64_ms / max(st64_n, 1)},
                      "split": {"value": value, "ms_per_step": ms32 / K, "rho_l2_vs_fp64": rho_l2,
                                "rho_linf_vs_fp64": rho_linf, "graph_replay_value": world * N * K / (gms32 / 1e3),
                                "stage_variant": variant32},
                      "split_over_fp64": value / value64},
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "stage_kernel (fused WENO5-char/LF sweeps + RK3 update)",
                         "alg_bytes_per_launch": alg_per_launch, "peak_kind": peak_kind,
                         "note": "FP64 and FP32 pipe bound, not HBM bound: ~13 kFLOP per cell-update"},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    exe = ROOT / "oracle" / "_ref" / "cbns3d_ref_inv"
    size = tuple(int(v) for v in a.size.split("x")) if a.size else None
    case, wl = make_case(a.case, size)
    metric = "cell-updates/s: learned-hybrid FP32 vs plain FP64 WENO5, same B200, rho-L2<=1e-5"
    if not exe.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cbns3d_ref_inv was not built "
                          "(the reference sources were absent at build time)"}))
        return
    K, W = a.steps, a.warmup
    N = n_updates(case)
    with tempfile.TemporaryDirectory() as td:
        base = Path(td)
        elapsed = {}
        for n in (W, W + K):
            d = case.write(base / f"run{n}", nsteps=n, checkpoint_freq=10 ** 9)
            r = subprocess.run([str(exe)], cwd=d, capture_output=True, text=True, timeout=1800)
            if r.returncode != 0:
                print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {r.stdout[-300:]}"}))
                return
            el = [float(l.split("=")[1]) for l in r.stdout.splitlines() if l.startswith("Elapsed Time")]
            elapsed[n] = el[-1]
    sec = max(elapsed[W + K] - elapsed[W], 1e-9)
    v = N * K / sec
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": v, "unit": "cell-updates/s", "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": 1e3 * sec / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl, "path": "reference CUDA build (FP64), its own executable and time loop",
                   "grid": list(case.shape), "cell_updates_per_step": N, "parallelism": "single GPU"},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                         "sample": f"{K} steps of the reference executable (GPU kernels, one host thread), "
                                   f"Elapsed Time of a {W + K}-step run minus a {W}-step run"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


if __name__ == "__main__":
    a = args()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
