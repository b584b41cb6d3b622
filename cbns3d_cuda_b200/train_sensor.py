"""Train the learned shock sensor and write its weights.

    python -m cbns3d_cuda_b200.train_sensor --out cbns3d_cuda_b200/data/sensor_weights.npz

writes the weights as .npz (parameters, tau, a JSON summary of the run) and as
the .bin file the C ABI and the host driver read (cbns_sensor_load_file).

Data: solver states of three flows, run with the split-precision path and
sampled every few steps: the isentropic vortex on the perturbed box (64 x 32 x
16), the spherical blast on the stretched, skewed box (96^3) and the Mach 1.2
shock / vortex interaction on the skewed channel (128 x 128 x 32).  Each
sampled face contributes its 15 features and its label (WENO5 weight
deviation > 0.05), both computed by the library (cbns_sensor_sample).

Training: Adam with a cosine learning-rate decay on the class-weighted
cross-entropy (cbns_mlp_grad and cbns_mlp_adam) over 90 % of the faces; the
held-out 10 % give recall and WENO5 fraction.

Threshold: a face takes the linear flux only when the network is confident
that it is smooth (p < tau); every other face -- confidently a shock face, or
one the network is unsure about -- takes WENO5.  tau is the lower edge of that
uncertainty band: at most 0.5 (the network's own decision boundary), low
enough that the held-out recall of WENO5-labelled faces is at least
--recall-floor, and calibrated in closed loop with WENO5 as the arbiter: on a
shock / vortex grid not used for training (192 x 192 x 96), 100 steps of the
hybrid flux (tcgen05 inference, as deployed) are compared with 100 steps of
the FP64 WENO5 path for each candidate tau, and the largest tau meeting all
three (its density L2 error at or below --l2-bound) is kept.
--recalibrate keeps the committed network and redoes only this choice.  Everything runs on the GPU; the script prints one line per stage and a
JSON summary, which is also stored in the output file.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import CBNS_Q, PREC_FP64, PREC_HYBRID, PREC_SPLIT, Block, cases, make_params, sensor


def _collect(case, nsteps, every, stride, log):
    import torch
    b = Block(make_params(*case.shape, **case.params, precision=PREC_SPLIT))
    b.calc_metrics(case.x, case.y, case.z)
    b.set_conservative(case.Q0)
    b.set_bc_calc_primitive(CBNS_Q)
    b.set_time(0.0)
    X, Y, D = [], [], []
    done = 0
    snap = 0
    while done <= nsteps:
        x, y, dv, _ = sensor.sample_faces(b, stride=stride, offset=snap % stride, with_dev=True)
        X.append(x.clone())
        Y.append(y.clone())
        D.append(dv.clone())
        snap += 1
        if done == nsteps:
            break
        n = min(every, nsteps - done)
        got = b.run(n, case.t_end)
        done += n
        if got < n:
            break
    b.close()
    X, Y, D = torch.cat(X), torch.cat(Y), torch.cat(D)
    log(f"{case.name} {case.shape}: {snap} snapshots, {X.shape[0]} faces, label-1 fraction {Y.float().mean().item():.4f}")
    return X, Y, D


def _rho(b, shape):
    IM, JM, KM = shape
    return b.get_conservative().reshape(KM + 4, JM + 4, IM + 4, 5)[2:-2, 2:-2, 2:-2, 0]


def calibrate(params, taus, nsteps, bound, log, shape=(192, 192, 96)):
    """Closed-loop threshold choice: density L2 error of the hybrid against
    FP64 WENO5 after nsteps for each tau (largest first)."""
    c = cases.case_shock_vortex(*shape)

    def run(precision, tau=None):
        b = Block(make_params(*c.shape, **c.params, precision=precision))
        b.calc_metrics(c.x, c.y, c.z)
        b.set_conservative(c.Q0)
        b.set_bc_calc_primitive(CBNS_Q)
        if tau is not None:
            b.sensor_load(params, tau)
        b.set_time(0.0)
        assert b.run(nsteps) == nsteps
        out = _rho(b, c.shape), (b.sensor_stats() if tau is not None else None)
        b.close()
        return out

    ref, _ = run(PREC_FP64)
    nref = float(np.sqrt(np.mean(ref ** 2)))
    rows = []
    for tau in sorted(taus, reverse=True):
        r, st = run(PREC_HYBRID, tau)
        l2 = float(np.sqrt(np.mean((r - ref) ** 2)) / nref)
        frac = st["weno_faces"] / (nsteps * st["faces_per_step"])
        rows.append(dict(tau=tau, rho_l2=l2, weno_fraction=frac, audit_fail_steps=st["audit_fail_steps"]))
        log(f"calibration tau {tau:g}: rho-L2 {l2:.3e}, WENO5 faces {frac:.4f}, "
            f"audit-rejected steps {st['audit_fail_steps']}")
    return rows


def choose_tau(rows, recall, bound, recall_floor, tau_max=0.5):
    """The largest candidate tau <= tau_max whose held-out recall (recall[tau])
    is at least recall_floor and whose closed-loop density L2 error is at most
    bound; the smallest candidate when none qualifies."""
    ok = [r for r in rows if r["tau"] <= tau_max and recall[r["tau"]] >= recall_floor and r["rho_l2"] <= bound]
    best = max(ok, key=lambda r: r["tau"]) if ok else min(rows, key=lambda r: r["tau"])
    return best["tau"]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default="cbns3d_cuda_b200/data/sensor_weights.npz")
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--l2-bound", type=float, default=1.0e-5)
    ap.add_argument("--taus", default="0.97,0.9,0.8,0.7,0.6,0.5,0.4,0.3,0.2,0.1,0.05,0.02")
    ap.add_argument("--recall-floor", type=float, default=0.95,
                    help="held-out recall of WENO5-labelled faces the threshold must keep")
    ap.add_argument("--recalibrate", action="store_true",
                    help="keep the network in --out and choose its threshold again")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--small", action="store_true", help="a quick run on smaller grids (for testing the script)")
    args = ap.parse_args(argv)
    import torch

    t0 = time.time()

    def log(msg):
        print(f"[{time.time() - t0:7.1f}s] {msg}", flush=True)

    if args.small:
        runs = [(cases.case_vortex(32, 16, 8), 20, 5, 1), (cases.case_blast(32, 32, 32), 20, 5, 2),
                (cases.case_shock_vortex(48, 48, 12), 20, 5, 2)]
    else:
        runs = [(cases.case_vortex(64, 32, 16), 100, 10, 1), (cases.case_blast(96, 96, 96), 150, 10, 4),
                (cases.case_shock_vortex(128, 128, 32), 200, 20, 2)]
    parts = [_collect(c, n, e, s, log) for c, n, e, s in runs]
    X = torch.cat([p[0] for p in parts])
    Y = torch.cat([p[1] for p in parts])
    n = X.shape[0]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(args.seed)
    perm = torch.randperm(n, device="cuda", generator=gen)
    nval = max(1, n // 10)
    vi, ti = perm[:nval], perm[nval:]
    Xt, Yt, Xv, Yv = X[ti].contiguous(), Y[ti].contiguous(), X[vi].contiguous(), Y[vi].contiguous()
    pos = float(Yt.float().mean().item())
    pos_weight = min(20.0, (1.0 - pos) / max(pos, 1e-6))
    if args.recalibrate:
        w = np.load(args.out)
        params = w["params"].astype(np.float32)
        prev = json.loads(str(w["summary"]))
        P = torch.from_numpy(params).cuda()
        hist, pos_weight = prev.get("loss_history"), prev.get("pos_weight")
        log(f"recalibrating the threshold of {args.out} (network kept)")
    else:
        log(f"training on {Xt.shape[0]} faces (label-1 fraction {pos:.4f}, pos_weight {pos_weight:.2f})")
        P, hist = sensor.train(Xt, Yt, epochs=args.epochs, batch=args.batch, lr=args.lr, pos_weight=pos_weight,
                               seed=args.seed, log=log, cosine=True)
        params = P.cpu().numpy().astype(np.float32)
    taus = [float(v) for v in args.taus.split(",")]
    if args.small:
        taus = taus[::3]
    pv = sensor.predict(P, Xv, tensor_cores=True)
    yb = Yv.bool()
    recall_of = {t: float(((pv >= t) & yb).sum().item() / max(1, int(yb.sum().item()))) for t in taus}
    weno_of = {t: float((pv >= t).float().mean().item()) for t in taus}
    for t in taus:
        log(f"held-out tau {t:g}: recall {recall_of[t]:.4f}, WENO5 fraction {weno_of[t]:.4f}")
    if args.small:
        rows = calibrate(params, taus, 20, args.l2_bound, log, shape=(48, 48, 16))
    else:
        rows = calibrate(params, taus, 100, args.l2_bound, log)
    for r in rows:
        r["val_recall"] = recall_of[r["tau"]]
    tau = choose_tau(rows, recall_of, args.l2_bound, args.recall_floor)
    summary = dict(faces=n, val_faces=nval, label_fraction=float(Yv.float().mean().item()), tau=tau,
                   val_recall=recall_of[tau], val_weno_fraction=weno_of[tau], recall_floor=args.recall_floor,
                   tau_rule="largest tau <= 0.5 with held-out recall >= recall_floor and closed-loop rho-L2 <= "
                            "l2_bound; faces with p >= tau (confident or uncertain) take WENO5",
                   calibration=rows, loss_history=hist, label_threshold=0.05, feature_scale=0.01,
                   cases=[f"{c.name} {c.shape} {ns} steps every {e} stride {s}" for c, ns, e, s in runs],
                   seed=args.seed, epochs=args.epochs, batch=args.batch, lr=args.lr, pos_weight=pos_weight)
    log(json.dumps(summary))
    np.savez(args.out, params=params, tau=np.float32(tau),
             summary=np.array(json.dumps(summary)))
    binp = str(args.out).rsplit(".", 1)[0] + ".bin"
    sensor.save_weights_bin(binp, params, tau)
    log(f"wrote {args.out} and {binp}")


if __name__ == "__main__":
    main()
