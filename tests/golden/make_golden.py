"""Generate the golden fixtures by running the reference itself.

Runs the unmodified reference executables built from the reference sources by
`make -C oracle ref` (oracle/_ref/cbns3d_ref_inv, oracle/_ref/cbns3d_ref_visc;
they need a GPU) on small seeded cases and stores, per case, the inputs (grid,
initial checkpoint or the free-stream flag, parameters), the per-step dt the
reference printed, and the checkpoint it wrote after the last step.

Cases avoid the reference's racy boundary branches: no wake cut
(i_begin = 1), whose mirror reads cross thread blocks, and KM % 4 != 1, so
that the k = KM-1 copy and its source k = KM-2 fall in the same 4-deep block
of the reference's boundary kernel.

Usage:  python tests/golden/make_golden.py [OUTDIR]   (default: tests/golden)
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cbns3d_cuda_b200 import cases  # noqa: E402

REF = ROOT / "oracle" / "_ref"


def golden_cases():
    """name -> (Case, nsteps).  Small grids keep the fixtures a few hundred kB."""
    out = {}
    c = cases.case_vortex(20, 14, 10)
    out["vortex_inviscid"] = (c, 20)

    c = cases.case_vortex(20, 14, 10)
    c.params = dict(c.params, i_begin=1, i_end=20)  # slip wall on the whole j = 0 face
    out["vortex_slipwall"] = (c, 12)

    c = cases.case_vortex(20, 14, 10)
    c.params = dict(c.params, i_begin=1, i_end=20, viscous=True, Re=200.0, T_inf=288.15)
    out["vortex_viscous_wall"] = (c, 10)

    c = cases.case_naca(32, 16, 6, first=1e-3)  # free-stream start (is_restart = 1), viscous, wall
    out["naca_viscous_freestream"] = (c, 10)
    return out


def run_reference(case, nsteps, workdir: Path):
    exe = REF / ("cbns3d_ref_visc" if case.params.get("viscous") else "cbns3d_ref_inv")
    if not exe.exists():
        raise SystemExit(f"{exe} missing: build it with `make -C oracle ref` where the reference sources are")
    case.write(workdir, nsteps=nsteps, checkpoint_freq=nsteps)
    r = subprocess.run([str(exe)], cwd=workdir, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    dts = []
    for line in r.stdout.splitlines():
        parts = [p.strip() for p in line.split(",")]
        # step lines are "n, dt, t"; the mesh-size line "IM, JM, KM" has no decimal point
        if len(parts) == 3 and any(ch in parts[1] for ch in ".eE"):
            try:
                int(parts[0])
                dts.append(float(parts[1]))
            except ValueError:
                pass
    t, Q = cases.read_checkpoint(workdir / "checkpoint.dat")
    return np.array(dts), t, Q


def main(outdir: Path):
    outdir.mkdir(parents=True, exist_ok=True)
    index = {}
    for name, (c, n) in golden_cases().items():
        with tempfile.TemporaryDirectory() as td:
            dts, t, Q = run_reference(c, n, Path(td))
        IM, JM, KM = c.shape
        np.savez_compressed(outdir / f"{name}.npz", x=c.x, y=c.y, z=c.z,
                            Q0=c.Q0 if c.Q0 is not None else np.zeros(0), dt=dts, t=t, Q=Q)
        index[name] = dict(shape=[IM, JM, KM], nsteps=n, params=c.params, t_end=c.t_end,
                           freestream_start=c.Q0 is None)
        print(f"{name}: {len(dts)} steps, t = {t:.6g}")
    (outdir / "index.json").write_text(json.dumps(index, indent=1, sort_keys=True))


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
