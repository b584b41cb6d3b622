#!/usr/bin/env python
"""Throughput of the RK3 right-hand-side path: cell-updates per second.

One step = one full SSP-RK3 step (sensor + audit for the hybrid, three fused
stage kernels, boundary conditions, device-side CFL dt) of one block of
synthetic input.  Default workload: the shock-vortex case of 256 x 256 x 128
nodes (inviscid; inputs larger than L2, so no flush is needed), W + K = 103
steps from the initial state.  A cell-update is one interior node advanced one
step; N_upd = (IM-2)(JM-2)(KM-2).

  value   device-resident throughput of the learned-sensor hybrid (per face
          WENO5-characteristic or linear upwind-5 flux in FP32, FP64 state,
          metrics and reductions), timed with CUDA events on the launch stream;
          its density L2 error against the plain FP64 path after the same steps
          is reported beside it and must stay <= 1e-5.
  paths   the same for the plain FP64 path (parity with the reference) and the
          split-precision path without the sensor (all faces WENO5 in FP32).
  e2e     the reference-style host-driven solve of the hybrid through the C
          ABI (block3d_cuda call sequence: dt read back every step, dt passed
          per stage), with the state uploaded from pinned host memory before
          and downloaded after the K steps inside the timed region; the same
          for the plain FP64 path under paths.fp64.e2e (the precision-matched
          end-to-end figure).
  paths.batch  the batched-blocks workload on the same GPU: 64 independent
          viscous blocks of uneven size (seeded draw), learned-sensor hybrid,
          one persistent stage launch per RK stage, per-block dt, W + K steps
          (--case batch runs it alone, beside the blocks stepped one by one).
  plain_vs_reference_linf  the plain FP64 path's state after the W + K steps
          against the reference's own CUDA build run on the same files for the
          same steps (largest relative L-inf over the five variables).
  roofline  HBM roofline of the dominant kernel (the fused stage kernel); the
          plain path's stage kernel also against the FP64 rate of a cuBLAS
          DGEMM measured in the same run.
  cpu_baseline  the FP64 CPU oracle (OpenMP, all host cores) on a bounded
          sample, with the host's CPU model.
  config  the workload alone (case, grid, cell-updates per step), the same
          in both arms' lines; how an arm computes it is under `path`.

--impl reference runs the reference's own build (oracle/_ref, compiled from its
sources) on the same case through its own executable and times it from its
"Elapsed Time" output (difference of a W-step and a (W+K)-step run, each
the shortest of two runs).

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
# FP64 FLOP the plain path executes per cell-update: dadd + dmul + 2 dfma
# counted by ncu over a stage-2 launch of the plain stage kernel (4,660 per
# node), times three stages
FP64_FLOP_PER_UPDATE = 13980.0
# nominal FP64 peak for context: 64 DFMA lanes per SM x 148 SMs x 2 FLOP x
# 1.965 GHz; the fraction is taken against the DGEMM rate measured in the run
FP64_NOMINAL_TFLOPS = 64 * 148 * 2 * 1.965e9 / 1e12
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per interior node
# of one stage-2 launch of the stage kernel, from single ncu captures on the
# shock-vortex case: plain FP64 kernel at 128x128x64, hybrid kernel at
# 192x192x96 (inputs larger than L2 in both); traffic grows with the nodes of
# a launch, so the figures scale to the bench grid
FP64_STAGE_DRAM_BYTES_PER_NODE = 240.0
HYBRID_STAGE_DRAM_BYTES_PER_NODE = 237.8


def args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="shock_vortex", choices=["shock_vortex", "blast", "vortex", "batch", "naca"])
    ap.add_argument("--blocks", type=int, default=64, help="--case batch: number of blocks (64 in the batched-blocks workload)")
    ap.add_argument("--no-one-by-one", action="store_true",
                    help="--case batch: skip stepping the same blocks one after the other")
    ap.add_argument("--size", default=None, help="IMxJMxKM (default: the case's config size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--to-tend", action="store_true",
                    help="run each path from the initial state to the case's end time (precision-form runs)")
    ap.add_argument("--t-end", type=float, default=None, help="--to-tend: end time (default: the case's)")
    ap.add_argument("--max-steps", type=int, default=100000, help="--to-tend: step limit")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-blocks pass of the default line")
    ap.add_argument("--no-reference-check", action="store_true",
                    help="skip the plain path's comparison with the reference build")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep each context's starting stage variant and k chunk (under a profiler the "
                         "autotuner's timings mean nothing)")
    ap.add_argument("--sensor", default=str(ROOT / "cbns3d_cuda_b200" / "data" / "sensor_weights.npz"))
    return ap.parse_args()


def replica_max(x, dist, torch, device):
    """The maximum of x over the ranks of the process group (x itself without one)."""
    if not dist:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(n_updates_per_step, steps, ms_max, world):
    """Whole-job cell-updates/s of `world` replicas, each advancing its own block
    of n_updates_per_step by `steps` steps, timed by the slowest rank (ms_max)."""
    return world * n_updates_per_step * steps / (ms_max / 1e3)


def make_case(name, size):
    from cbns3d_cuda_b200 import cases
    if name == "shock_vortex":
        IM, JM, KM = size or (256, 256, 128)
        return cases.case_shock_vortex(IM, JM, KM), f"shock-vortex {IM}x{JM}x{KM}, inviscid"
    if name == "blast":
        IM, JM, KM = size or (384, 384, 384)
        return cases.case_blast(IM, JM, KM), f"spherical blast {IM}x{JM}x{KM}, inviscid"
    if name == "naca":
        P, JM, KM = size or (384, 128, 4)
        c = cases.case_naca_ogrid(P, JM, KM, grid="marched", start="potential")
        return c, (f"NACA 0012 O-grid {P}x{JM}x{KM} (+{2 * 4} wrap points), viscous, M 0.8, AoA 1.25, Re 5e4, "
                   f"first cell 1e-5, CFL 0.8, potential-flow start")
    IM, JM, KM = size or (64, 32, 16)
    return cases.case_vortex(IM, JM, KM), f"isentropic vortex {IM}x{JM}x{KM}, inviscid"


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


SENSOR = None  # (params, tau) of the trained sensor network
NO_AUTOTUNE = False  # --no-autotune: keep each context's starting stage variant
REF_REPEATS = 2  # --impl reference: runs per step count (the shortest is kept)


def load_sensor(path):
    global SENSOR
    w = np.load(path)
    SENSOR = (w["params"].astype(np.float32), float(w["tau"]))
    return SENSOR


def init_block(case, precision):
    from cbns3d_cuda_b200 import CBNS_Q, PREC_HYBRID, Block, make_params
    p = dict(case.params)
    p["precision"] = precision
    b = Block(make_params(*case.shape, **p))
    b.calc_metrics(case.x, case.y, case.z)
    if case.Q0 is None:
        b.initial_condition()
        b.calc_conservative(CBNS_Q)
    else:
        b.set_conservative(case.Q0)
        if p.get("viscous"):
            b.calc_primitive(CBNS_Q)
    b.set_bc_calc_primitive(CBNS_Q)
    if p.get("viscous"):
        b.calc_viscous_terms()
    if precision == PREC_HYBRID:
        b.sensor_load(*SENSOR)
    return b


def workload_config(wl, case, n):
    """The `config` of both arms' lines: the workload alone (how each arm
    computes it goes under `path`)."""
    return {"workload": wl, "grid": list(case.shape), "cell_updates_per_step": n,
            "l2": "inputs larger than L2 (the grid's state and metric arrays)"}


def n_updates(case):
    IM, JM, KM = case.shape
    return (IM - 2) * (JM - 2) * (KM - 2)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def device_pass(case, precision, K, W, torch, dist, clocks=None, keep_state=False):
    """W untimed steps, K steps replayed from the CUDA graph and timed with
    events on the launch stream (optionally with clock sampling), the state
    read back, then K more steps with events around every kernel for the
    per-kernel breakdown.  Returns a dict."""
    from cbns3d_cuda_b200 import PREC_HYBRID
    b = init_block(case, precision)
    stream = torch.cuda.Stream()  # a real stream: the legacy default stream cannot be graph-captured
    b.set_stream(stream.cuda_stream)
    if NO_AUTOTUNE:  # the context's own starting variant and k chunk
        out = {"variant": None}
    else:
        out = {"variant": b.autotune()}
    out["kchunk"] = b.stage_kchunk()
    b.set_time(0.0)
    b.run(W)
    if precision == PREC_HYBRID:
        b.sensor_stats_reset()
    l0 = b.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if clocks:
        clocks.__enter__()
    e0.record(stream)
    b.run_async(K)
    e1.record(stream)
    torch.cuda.synchronize()
    if clocks:
        clocks.__exit__(None, None, None)
    if dist:
        dist.barrier()
    out["ms"] = e0.elapsed_time(e1)
    out["launches"] = b.launch_count() - l0
    IM, JM, KM = case.shape
    q = b.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)
    out["rho"] = q[2:-2, 2:-2, 2:-2, 0].copy()
    if keep_state:
        out["q"] = q
    out["stats"] = b.sensor_stats() if precision == PREC_HYBRID else None
    b.prof_enable(True)
    b.prof_reset()
    b.run(K)
    out["kern"] = {kid: b.prof_read(kid) for kid in range(7)}
    b.prof_enable(False)
    b.close()
    return out


def e2e_pass(case, K, torch, precision):
    """Host-driven solve through the C ABI with host buffers (pinned): the
    state uploaded, K steps of the reference's time loop (dt read back every
    step), the state downloaded, all inside the timed region."""
    from cbns3d_cuda_b200 import CBNS_Q, _abi
    b = init_block(case, precision)
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


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def fp64_peak_tflops(torch):
    """FP64 rate of a cuBLAS DGEMM (torch.matmul, 8192^3, best of 5, CUDA events)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def reference_state(case, nsteps, timeout=1800):
    """The reference build's conservative state (ghosted AoS, as its checkpoint
    stores it) after nsteps steps of the case, or None when it was not built."""
    exe = ROOT / "oracle" / "_ref" / "cbns3d_ref_inv"
    if not exe.exists():
        return None
    from cbns3d_cuda_b200 import cases
    with tempfile.TemporaryDirectory() as td:
        d = case.write(Path(td) / "run", nsteps=nsteps, checkpoint_freq=nsteps)
        r = subprocess.run([str(exe)], cwd=d, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed: {r.stdout[-300:]}")
        return cases.read_checkpoint(d / "checkpoint.dat")[1]


def cpu_baseline(case, budget_s=10.0, max_steps=100):
    """The FP64 oracle on the host cores: whole RK3 steps of the case until
    about budget_s seconds of CPU work (at most max_steps)."""
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
        if el >= budget_s or steps >= max_steps:
            break
    o.close()
    return {"value": n_updates(case) * steps / el, "unit": "cell-updates/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "nproc": cores, "cpu_model": cpu_model(),
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
    from cbns3d_cuda_b200 import PREC_FP64, PREC_HYBRID, PREC_SPLIT
    load_sensor(a.sensor)
    size = tuple(int(v) for v in a.size.split("x")) if a.size else None
    case, wl = make_case(a.case, size)
    K, W = a.steps, a.warmup
    N = n_updates(case)
    IM, JM, KM = case.shape

    # plain FP64 path, the split path without the sensor, then the
    # learned-sensor hybrid (headline) with clocks sampled during its timed region
    p64 = device_pass(case, PREC_FP64, K, W, torch, dist, keep_state=not a.no_reference_check)
    p32 = device_pass(case, PREC_SPLIT, K, W, torch, dist)
    clk = Clocks(local)
    ph = device_pass(case, PREC_HYBRID, K, W, torch, dist, clocks=clk)
    clocks = clk.summary()
    r64, r32, rh = p64["rho"], p32["rho"], ph["rho"]
    ms64, ms32, msh = p64["ms"], p32["ms"], ph["ms"]
    kern64, kern32, kernh = p64["kern"], p32["kern"], ph["kern"]
    stats, launches = ph["stats"], ph["launches"]
    variant32, varianth = p32["variant"], ph["variant"]

    def err(r):
        return (float(np.sqrt(np.mean((r - r64) ** 2) / np.mean(r64 ** 2))),
                float(np.max(np.abs(r - r64)) / np.max(np.abs(r64))))

    l2_32, linf_32 = err(r32)
    l2_h, linf_h = err(rh)

    def reduce_max(x):
        return replica_max(x, dist, torch, "cuda")

    ms32, ms64, msh = reduce_max(ms32), reduce_max(ms64), reduce_max(msh)
    value = replica_throughput(N, K, msh, world)
    value32 = replica_throughput(N, K, ms32, world)
    value64 = replica_throughput(N, K, ms64, world)

    e2e = e2e64 = None
    if not a.no_e2e:
        ems, eb = e2e_pass(case, K, torch, PREC_HYBRID)
        ems = reduce_max(ems)
        e2e = {"value": replica_throughput(N, K, ems, world), "unit": "cell-updates/s", **eb}
        ems, eb = e2e_pass(case, K, torch, PREC_FP64)
        ems = reduce_max(ems)
        e2e64 = {"value": replica_throughput(N, K, ems, world), "unit": "cell-updates/s", **eb}

    peak, peak_kind = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch)
    # the per-kernel events come from a second run of K steps (same work per step)
    st_ms, st_n = kernh[0]
    alg_per_launch = ALG_BYTES_PER_UPDATE / 3.0 * N
    achieved = alg_per_launch / (st_ms / st_n / 1e3) / 1e9 if st_n else None
    traffic = HYBRID_STAGE_DRAM_BYTES_PER_NODE * N
    traffic64 = FP64_STAGE_DRAM_BYTES_PER_NODE * N
    # the plain path's stage kernel: HBM and FP64-pipe fractions
    st64_ms, st64_n = kern64[0]
    st64_launch_s = st64_ms / max(st64_n, 1) / 1e3
    ach64 = alg_per_launch / st64_launch_s / 1e9 if st64_n else None
    tfl64 = FP64_FLOP_PER_UPDATE / 3.0 * N / st64_launch_s / 1e12 if st64_n else None

    # the batched-blocks workload on this GPU (64 viscous blocks, hybrid)
    batch = None
    if not a.no_batch:
        batch = batch_pass(a.blocks, K, W, torch, one_by_one=False)
        batch.pop("shapes")
        bms = reduce_max(batch["ms_per_step"] * K)
        batch["ms_per_step"] = bms / K
        batch["value"] = replica_throughput(batch["cell_updates_per_step"], K, bms, world)

    # the plain path against the reference's own build after the same W + K
    # steps of the same case: relative L-inf per conservative variable
    ref_cmp = None
    if not a.no_reference_check and rank == 0:
        qr = reference_state(case, W + K)
        if qr is not None:
            q64 = p64["q"]
            per = [float(np.max(np.abs(q64[..., n] - qr[..., n])) / np.max(np.abs(qr[..., n]))) for n in range(5)]
            ref_cmp = {"linf_per_variable": per, "max": max(per), "steps": W + K,
                       "what": "plain FP64 path vs the reference CUDA build (oracle/_ref/cbns3d_ref_inv), same "
                               "grid file, initial checkpoint and input.txt; relative L-inf over the ghosted box"}

    def kern_ms(k):
        return {name: {"ms_per_step": k[i][0] / K, "groups_per_step": k[i][1] / K}
                for i, name in enumerate(["stage", "bc", "viscous", "dt", "sensor", "audit", "weno_faces"]) if k[i][1]}

    weno_frac = stats["weno_faces"] / (K * stats["faces_per_step"]) if stats["faces_per_step"] else None
    if rank == 0:
        cpu = None if (a.no_cpu_baseline or world > 1) else cpu_baseline(case)  # rank 0 at N = 1 only
        line = {
            "metric": "cell-updates/s: learned-hybrid FP32 vs plain FP64 WENO5, same B200, rho-L2<=1e-5",
            "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": msh / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 flux / f64 state", "data": "synthetic",
            "config": workload_config(wl, case, N),
            "path": "learned-sensor hybrid: per face WENO5-char or linear upwind-5 flux (FP32), "
                    "FP64 state, metrics, dt; sensor MLP on tcgen05 (BF16) every 3rd step, decisions "
                    "held and widened in between; audit every step on a rotating 1/97 sample of the "
                    "linear faces",
            "parallelism": f"replicas x{world}",
            "sensor": {"weights": os.path.relpath(a.sensor, ROOT), "tau": SENSOR[1]},
            "rho_l2_vs_fp64": l2_h, "rho_linf_vs_fp64": linf_h,
            "plain_vs_reference_linf": ref_cmp["max"] if ref_cmp else None,
            "paths": {"fp64": {"value": value64, "ms_per_step": ms64 / K, "stage_variant": p64["variant"], "stage_kchunk": p64["kchunk"],
                               "kernels": kern_ms(kern64),
                               "roofline_hbm": {"achieved": ach64, "peak": peak, "unit": "GB/s",
                                                "frac": (ach64 / peak) if ach64 else None, "traffic": traffic64},
                               "roofline_fp64": {"achieved": tfl64, "peak": fp64_peak, "unit": "TFLOP/s",
                                                 "frac": (tfl64 / fp64_peak) if tfl64 else None,
                                                 "flop_per_update": FP64_FLOP_PER_UPDATE,
                                                 "peak_kind": "measured in this run: cuBLAS DGEMM 8192^3",
                                                 "nominal": FP64_NOMINAL_TFLOPS},
                               "e2e": e2e64, "plain_vs_reference": ref_cmp},
                      "split": {"value": value32, "ms_per_step": ms32 / K, "rho_l2_vs_fp64": l2_32,
                                "rho_linf_vs_fp64": linf_32, "stage_variant": variant32, "stage_kchunk": p32["kchunk"],
                                "kernels": kern_ms(kern32)},
                      "hybrid": {"value": value, "ms_per_step": msh / K, "rho_l2_vs_fp64": l2_h,
                                 "rho_linf_vs_fp64": linf_h, "weno_face_fraction": weno_frac,
                                 "audit_rejected_steps": stats["audit_fail_steps"],
                                 "audit_faces": stats["audit_faces"], "audit_max_rel_diff": stats["audit_max"],
                                 "sensor_timeouts": stats["sensor_fail"], "stage_variant": varianth, "stage_kchunk": ph["kchunk"],
                                 "kernels": kern_ms(kernh)},
                      "batch": batch,
                      "hybrid_over_fp64": value / value64, "hybrid_over_split": value / value32},
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "stage_kernel, hybrid (linear upwind-5/LF faces, WENO5 faces read from the WENO5-face pass, RK3 update)",
                         "alg_bytes_per_launch": alg_per_launch, "peak_kind": peak_kind,
                         "note": "load-latency and issue bound, not HBM bound"},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def ref_loop_seconds(runs, W, K):
    """Seconds of K reference steps: the shortest time loop of the (W+K)-step
    runs minus the shortest of the W-step runs (runs: step count -> the
    Elapsed Time of each run)."""
    elapsed = {n: min(v) for n, v in runs.items()}
    return max(elapsed[W + K] - elapsed[W], 1e-9)


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
    # each step count runs REF_REPEATS times and keeps its shortest time loop:
    # the reference's calc_dt allocates through thrust on every step, and its
    # loop time varies from run to run (30-46 ms per step seen on this grid)
    runs = {}
    with tempfile.TemporaryDirectory() as td:
        base = Path(td)
        for n in (W, W + K):
            d = case.write(base / f"run{n}", nsteps=n, checkpoint_freq=10 ** 9)
            for _ in range(REF_REPEATS):
                r = subprocess.run([str(exe)], cwd=d, capture_output=True, text=True, timeout=1800)
                if r.returncode != 0:
                    print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {r.stdout[-300:]}"}))
                    return
                el = [float(l.split("=")[1]) for l in r.stdout.splitlines() if l.startswith("Elapsed Time")]
                runs.setdefault(n, []).append(el[-1])
    sec = ref_loop_seconds(runs, W, K)
    v = N * K / sec
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": v, "unit": "cell-updates/s", "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": 1e3 * sec / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(wl, case, N),
        "path": "reference CUDA build (FP64), its own executable and time loop", "parallelism": "single GPU",
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                         "sample": f"{K} steps of the reference executable (GPU kernels, one host thread), "
                                   f"Elapsed Time of a {W + K}-step run minus a {W}-step run, each the "
                                   f"shortest of {REF_REPEATS} runs"},
        "elapsed_s": {str(n): v for n, v in runs.items()},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_to_tend(a):
    """A case run from its initial state to its end time on each path (plain
    FP64, split, learned-sensor hybrid), as the precision-form configuration
    asks: density L2 / L-inf of the FP32-flux paths against the FP64 run at
    the same end time, and each path's throughput over the whole run (CUDA
    events on the launch stream, steps enqueued from the graph in chunks,
    host reads of the step counter between chunks inside the timed region)."""
    import torch
    from cbns3d_cuda_b200 import PREC_FP64, PREC_HYBRID, PREC_SPLIT
    torch.cuda.set_device(0)
    load_sensor(a.sensor)
    size = tuple(int(v) for v in a.size.split("x")) if a.size else None
    case, wl = make_case(a.case, size)
    N = n_updates(case)
    t_end = case.t_end if a.t_end is None else a.t_end
    chunk = 50
    res = {}
    clocks = None
    for name, prec in (("fp64", PREC_FP64), ("split", PREC_SPLIT), ("hybrid", PREC_HYBRID)):
        b = init_block(case, prec)
        stream = torch.cuda.Stream()
        b.set_stream(stream.cuda_stream)
        variant = None if NO_AUTOTUNE else b.autotune()
        b.set_time(0.0)
        if prec == PREC_HYBRID:
            b.sensor_stats_reset()
        clk = Clocks(0) if prec == PREC_HYBRID else None
        torch.cuda.synchronize()
        if clk:
            clk.__enter__()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        steps = 0
        while True:
            n = b.run(chunk, t_end)
            steps += n
            if n < chunk or steps >= a.max_steps:
                break
        e1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__(None, None, None)
            clocks = clk.summary()
        ms = e0.elapsed_time(e1)
        t_fin, dt_last = b.get_time()
        IM, JM, KM = case.shape
        rho = b.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)[2:-2, 2:-2, 2:-2, 0].copy()
        stats = b.sensor_stats() if prec == PREC_HYBRID else None
        b.close()
        res[name] = {"value": N * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps, "t_final": t_fin,
                     "stage_variant": variant, "rho": rho, "stats": stats}
        del b
    r64 = res["fp64"]["rho"]
    out_paths = {}
    for name, r in res.items():
        d = {k: v for k, v in r.items() if k not in ("rho", "stats")}
        if name != "fp64":
            rr = r["rho"]
            d["rho_l2_vs_fp64"] = float(np.sqrt(np.mean((rr - r64) ** 2) / np.mean(r64 ** 2)))
            d["rho_linf_vs_fp64"] = float(np.max(np.abs(rr - r64)) / np.max(np.abs(r64)))
        if r["stats"]:
            st = r["stats"]
            d["weno_face_fraction"] = st["weno_faces"] / max(1, r["steps"] * st["faces_per_step"])
            d["audit_rejected_steps"] = st["audit_fail_steps"]
            d["sensor_timeouts"] = st["sensor_fail"]
        out_paths[name] = d
    h = out_paths["hybrid"]
    print(json.dumps({
        "metric": "cell-updates/s: learned-hybrid FP32 vs plain FP64 WENO5, same B200, rho-L2<=1e-5",
        "value": h["value"], "unit": "cell-updates/s", "n_gpus": 1, "steps": h["steps"], "warmup": 0,
        "ms_per_step": h["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 flux / f64 state", "data": "synthetic",
        "config": {"workload": f"{wl}, from the initial state to t = {t_end}", "grid": list(case.shape),
                   "cell_updates_per_step": N, "t_end": t_end,
                   "l2": "inputs larger than L2"},
        "rho_l2_vs_fp64": h["rho_l2_vs_fp64"], "rho_linf_vs_fp64": h["rho_linf_vs_fp64"],
        "paths": out_paths, "hybrid_over_fp64": h["value"] / out_paths["fp64"]["value"],
        "split_over_fp64": out_paths["split"]["value"] / out_paths["fp64"]["value"],
        "clocks": clocks}))


def run_naca(a):
    """The viscous NACA 0012 O-grid configuration on the plain FP64 path: K
    steps from the started flow (graph replays in chunks of 500, each timed
    with CUDA events on the launch stream), the state checked for positivity
    after every chunk (outside the timed region), and the per-kernel times of
    one more chunk."""
    import torch
    from cbns3d_cuda_b200 import PREC_FP64
    torch.cuda.set_device(0)
    size = tuple(int(v) for v in a.size.split("x")) if a.size else None
    case, wl = make_case("naca", size)
    IM, JM, KM = case.shape
    N = n_updates(case)
    b = init_block(case, PREC_FP64)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    b.set_time(0.0)
    K = a.steps
    chunk = min(500, K)
    ms_total, done, history = 0.0, 0, []
    clk = Clocks(0)
    clk.__enter__()
    while done < K:
        n = min(chunk, K - done)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run_async(n)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_total += e0.elapsed_time(e1)
        done += n
        q = b.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)[2:-2, 2:-2, 2:-2]
        r = q[..., 0]
        pr = 0.4 * (q[..., 4] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2 + q[..., 3] ** 2) / r)
        t, dt = b.get_time()
        history.append({"steps": done, "t": t, "dt": dt, "rho_min": float(np.min(r)), "p_min": float(np.min(pr)),
                        "p_max": float(np.max(pr)), "finite": bool(np.isfinite(q).all())})
        if not history[-1]["finite"] or history[-1]["p_min"] <= 0 or history[-1]["rho_min"] <= 0:
            break
    clk.__exit__(None, None, None)
    b.prof_enable(True)
    b.prof_reset()
    b.run(100)
    kern = {name: {"ms_per_step": b.prof_read(i)[0] / 100, "groups_per_step": b.prof_read(i)[1] / 100}
            for i, name in enumerate(["stage", "bc", "viscous", "dt", "sensor", "audit", "weno_faces"])
            if b.prof_read(i)[1]}
    b.close()
    ok = all(h["finite"] and h["p_min"] > 0 and h["rho_min"] > 0 for h in history)
    print(json.dumps({
        "metric": "cell-updates/s: learned-hybrid FP32 vs plain FP64 WENO5, same B200, rho-L2<=1e-5",
        "value": N * done / (ms_total / 1e3), "unit": "cell-updates/s", "n_gpus": 1, "steps": done, "warmup": 0,
        "ms_per_step": ms_total / done, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl, "path": "plain FP64 (viscous divergence at the node, full viscous dt limit, "
                                           "O-grid boundary mode)", "grid": list(case.shape),
                   "cell_updates_per_step": N},
        "stable": ok, "history": history, "kernels": kern, "clocks": clk.summary()}))


def batch_pass(nblocks, K, W, torch, one_by_one=True, clocks=None):
    """The batched-blocks workload: independent viscous blocks of uneven size
    (seeded draw), learned-sensor hybrid, advanced by one persistent
    work-queue launch of the stage kernel per RK stage (cbns_batch_run) with
    per-block dt; optionally beside it the same blocks stepped one after the
    other on the same stream (one CUDA graph per block).  Both timed with CUDA
    events on that stream.  Returns a dict."""
    from cbns3d_cuda_b200 import CBNS_Q, PREC_HYBRID, Batch, Block, cases, make_params
    cs, draw = cases.case_batch(nblocks, seed=0)
    N = sum((c.shape[0] - 2) * (c.shape[1] - 2) * (c.shape[2] - 2) for c in cs)

    def make():
        out = []
        for c in cs:
            b = Block(make_params(*c.shape, **c.params, precision=PREC_HYBRID))
            b.calc_metrics(c.x, c.y, c.z)
            b.set_conservative(c.Q0)
            b.calc_primitive(CBNS_Q)
            b.set_bc_calc_primitive(CBNS_Q)
            b.calc_viscous_terms()
            b.sensor_load(*SENSOR)
            b.set_time(0.0)
            out.append(b)
        return out

    stream = torch.cuda.Stream()  # every launch of both passes goes to this stream

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    blocks = make()
    bt = Batch(blocks, stream.cuda_stream)
    bt.run(W)
    if clocks:
        clocks.__enter__()
    ms_batch = timed(lambda: bt.run_async(K))
    if clocks:
        clocks.__exit__(None, None, None)
    bt.close()
    for b in blocks:
        b.close()
    out = {"value": N * K / (ms_batch / 1e3), "ms_per_step": ms_batch / K, "steps": K, "blocks": len(cs),
           "cell_updates_per_step": N, "shapes": [d["shape"] for d in draw],
           "workload": f"batched blocks: {len(cs)} viscous blocks, sizes 32^3..128x64x64 (seed 0), Mach U[0.3,2], "
                       "Re U[1e3,1e5], far-field boundaries, learned-sensor hybrid, per-block dt"}
    if one_by_one:
        blocks = make()
        for b in blocks:
            b.set_stream(stream.cuda_stream)
            b.run(W)

        def alone():
            for b in blocks:
                b.run_async(K)

        ms_alone = timed(alone)
        for b in blocks:
            b.close()
        out["blocks_one_by_one"] = {"value": N * K / (ms_alone / 1e3), "ms_per_step": ms_alone / K}
        out["batch_over_one_by_one"] = ms_alone / ms_batch
    return out


def run_batch(a):
    """The batched-blocks workload alone, as its own bench line (batch_pass)."""
    import torch
    torch.cuda.set_device(0)
    load_sensor(a.sensor)
    clk = Clocks(0)
    r = batch_pass(a.blocks, a.steps, a.warmup, torch, one_by_one=not a.no_one_by_one, clocks=clk)
    print(json.dumps({
        "metric": "cell-updates/s: learned-hybrid FP32 vs plain FP64 WENO5, same B200, rho-L2<=1e-5",
        "value": r["value"], "unit": "cell-updates/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 flux / f64 state", "data": "synthetic",
        "config": {"workload": r["workload"], "cell_updates_per_step": r["cell_updates_per_step"],
                   "blocks": r["blocks"], "shapes": r["shapes"]},
        "paths": {"batch": {"value": r["value"], "ms_per_step": r["ms_per_step"]},
                  "blocks_one_by_one": r.get("blocks_one_by_one"),
                  "batch_over_one_by_one": r.get("batch_over_one_by_one")},
        "clocks": clk.summary(),
    }))


if __name__ == "__main__":
    a = args()
    NO_AUTOTUNE = a.no_autotune
    if a.impl == "reference":
        run_reference(a)
    elif a.case == "batch":
        run_batch(a)
    elif a.case == "naca":
        run_naca(a)
    elif a.to_tend:
        run_to_tend(a)
    else:
        run_ours(a)
