"""Train the learned subgrid closure on the dynamic procedure's Cs^2.

    python -m freeshearlayer_b200.train_closure --out freeshearlayer_b200/closure_weights.f32

Runs temporal shear layers on the GPU (FP32 bulk, dynamic Smagorinsky) at
convective Mach 0.3, 0.5 and 0.7 (box 2pi x pi x pi), each
GRID:AMP:STEPS:RE entry of --runs once per Mach number:
  - velocity noise of 1e-3 dU at Re_dw0 1000 on the 256x128x128 and the
    512x256x256 grid (the laminar phase the production runs start in);
  - noise of 5e-2 dU at Re_dw0 2e4 on a 128x64x64 and a 256x128x128 grid,
    run through the roll-up into turbulence, where the dynamic SGS viscosity
    reaches and passes the molecular one.
Every 50 steps it harvests (features, dynamic Cs^2) samples, with a cell
stride per run that spreads the --samples budget over all snapshots, trains
the MLP with Adam on the tensor-core kernels and writes the FP32 parameter
vector (FSL_CLOSURE_NPARAMS little-endian floats).  Finally it judges the
trained closure on fresh runs (another Mach number and seed) and prints one
JSON log line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "closure_weights.f32")


def shear_params(grid, Mc, Re=1000.0, precision=1):
    L, H, D = grid
    dU = 2.0 * Mc * math.sqrt(1.4 * 1e5 / 1.0)
    return dict(LEN=L, HIG=H, DEP=D, deltaX=2 * math.pi / L, deltaY=math.pi / H, deltaZ=math.pi / D,
                deltaT=1e-5, Answer=0, numstep=0, mu_L=dU * 1.0 / Re, Pr_L=0.72, Pr_T=0.8, Cs=0.01,
                BL_HIG=0, Ua=0.0, Va=0.0, Wa=0.0, Ns_min=10, Nst=50, f_step=50, nStages=3,
                maxCoNum=0.5, setup=1, cfl_mode=1, seed_X=0.317391239817, precision=precision,
                sgs=0, recon=0), dU


def load_weights(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    w = np.fromfile(path, dtype="<f4")
    if w.size != 9473:
        raise ValueError("%s: expected 9473 float32 parameters, found %d" % (path, w.size))
    return w


def judge(fsl, w, grid, Mc, amp, steps, seed, Re=1000.0):
    p, dU = shear_params(grid, Mc, Re)
    state, _ = fsl.temporal_state(p, Mc, 1.0, amp, seed)
    d = fsl.Domain(p)
    d.upload_state(state)
    d.closure_set_scales(1.0 / dU, 1.0)
    d.closure_set_weights(w)
    if steps:
        d.step(steps)
    st = d.closure_compare()
    d.close()
    return {"grid": list(grid), "Mc": Mc, "Re": Re, "amp": amp, "steps": steps, "cs2_profile_err": st.profile_err,
            "cs2_cell_err": st.cell_err, "mu_profile_err": st.mu_profile_err, "visc_err": st.visc_err,
            "mu_active_err": st.mu_active_err, "dyn_ratio": st.dyn_ratio, "active_rows": st.active_rows}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--runs", default="256x128x128:0.001:2000:1000,512x256x256:0.001:600:1000,"
                                      "128x64x64:0.05:12000:20000,256x128x128:0.05:20000:20000")
    ap.add_argument("--mach", default="0.3,0.5,0.7")
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--samples", type=float, default=2e8, help="target number of harvested samples")
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=20251203)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(HERE))
    import freeshearlayer_b200 as fsl

    runs = []
    for r in args.runs.split(","):
        f = r.split(":")
        runs.append((tuple(int(x) for x in f[0].split("x")), float(f[1]), int(f[2]),
                     float(f[3]) if len(f) > 3 else 1000.0))
    machs = [float(m) for m in args.mach.split(",")]
    nsnap = sum(len(machs) * (steps // args.every + 1) for _, _, steps, _ in runs)
    per_snap = args.samples / nsnap
    tr = fsl.Trainer(int(args.samples * 1.1) + 1, seed=args.seed)
    log = {"runs": []}
    t0 = time.time()
    for grid, amp, steps, Re in runs:
        band = (grid[0] - 4) * (grid[1] - 4) * (grid[2] - 4)
        stride = max(1, int(math.ceil(band / per_snap)))
        for Mc in machs:
            p, dU = shear_params(grid, Mc, Re)
            state, _ = fsl.temporal_state(p, Mc, 1.0, amp, args.seed + int(Mc * 10) + int(amp * 1e4))
            d = fsl.Domain(p)
            d.upload_state(state)
            d.closure_set_scales(1.0 / dU, 1.0)
            tr.harvest(d, stride)
            for _ in range(steps // args.every):
                d.step(args.every)
                tr.harvest(d, stride)
            log["runs"].append({"grid": list(grid), "Mc": Mc, "Re": Re, "amp": amp, "steps": steps,
                                "stride": stride, "samples": tr.size})
            print("harvest %s Mc %.1f Re %g amp %g stride %d -> %d samples (%.0f s)" % (
                grid, Mc, Re, amp, stride, tr.size, time.time() - t0), flush=True)
            d.close()
    X, Y = tr.samples(min(tr.size, 1 << 20))
    p0 = tr.weights()
    p0[9472] = float(np.mean(Y))
    tr.set_weights(p0)
    _, loss0 = tr.gradient()
    t1 = time.time()
    loss = tr.train(epochs=args.epochs, batch=args.batch, lr=args.lr)
    t2 = time.time()
    w = tr.weights()
    w.astype("<f4").tofile(args.out)
    log.update({"samples": tr.size, "loss0": loss0, "loss": loss, "epochs": args.epochs,
                "batch": args.batch, "lr": args.lr, "train_s": t2 - t1,
                "samples_per_s": tr.size * args.epochs / max(t2 - t1, 1e-9)})
    # the trained closure against the dynamic procedure on fresh runs
    s = args.seed + 99
    log["judge"] = [judge(fsl, w, (512, 256, 256), 0.7, 1e-3, 0, s), judge(fsl, w, (512, 256, 256), 0.7, 1e-3, 300, s)]
    for steps in (0, 4000, 8000, 10000):  # Mc 0.6: not a training Mach number
        log["judge"].append(judge(fsl, w, (128, 64, 64), 0.6, 0.05, steps, s, Re=20000.0))
    print(json.dumps(log), flush=True)


if __name__ == "__main__":
    main()
