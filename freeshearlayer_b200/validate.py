"""Long-run comparisons of the step's variants on one GPU.

    python -m freeshearlayer_b200.validate --config c2 [--steps 2000]
    python -m freeshearlayer_b200.validate --config c5 [--steps 5000]

c2: temporal shear layer 256x128x128, Mc 0.6, Re_dw0 1000: the plain FP64
    path (dynamic Smagorinsky, bit-identical to the CPU oracle at small
    sizes), FP32 bulk with the FP32 dynamic procedure, and both again with
    PPM reconstruction, from the same seeded state.
c5: 512x256x256, Mc 0.7, Re_dw0 1000: the plain FP64 path against FP32 bulk +
    the learned closure (judged every 100 steps), and both again with PPM.
turb: 256x128x128, Mc 0.6, Re_dw0 2e4, noise 5e-2 dU, 20000 steps through
    the roll-up into turbulence: the SGS models against each other
    (freeshearlayer_b200/closure_gain.py).

Each lower-precision arm is compared with the FP64 arm of the same
reconstruction; FP64 PPM is also compared with the plain FP64 path (the
difference of the schemes, not an error).

Box 2pi x pi x pi, acoustic CFL 0.5, velocity noise 1e-3 dU (seed 20251203).
Every --every steps each arm records its momentum thickness; at the end the
relative L2 of each conserved variable against the FP64 arm, the momentum
thickness growth and the Favre Reynolds-stress profiles are compared.  One
JSON line per arm, then a summary line.
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

CONFIGS = {
    "c2": dict(grid=(256, 128, 128), Mc=0.6, Re=1000.0, steps=2000,
               arms=[("fp64-dynamic", 0, 0, 0), ("fp32-dynamic", 1, 0, 0), ("fp64-ppm", 0, 0, 1),
                     ("fp32-dynamic-ppm", 1, 0, 1)],
               pairs=[("fp32-dynamic", "fp64-dynamic"), ("fp32-dynamic-ppm", "fp64-ppm"),
                      ("fp64-ppm", "fp64-dynamic")]),
    "c5": dict(grid=(512, 256, 256), Mc=0.7, Re=1000.0, steps=5000,
               arms=[("fp64-dynamic", 0, 0, 0), ("fp32-learned", 1, 1, 0), ("fp64-ppm", 0, 0, 1),
                     ("fp32-learned-ppm", 1, 1, 1)],
               pairs=[("fp32-learned", "fp64-dynamic"), ("fp32-learned-ppm", "fp64-ppm"),
                      ("fp64-ppm", "fp64-dynamic")]),
}


def params(grid, Mc, Re, precision, sgs, recon):
    L, H, D = grid
    dU = 2.0 * Mc * math.sqrt(1.4 * 1e5 / 1.0)
    return dict(LEN=L, HIG=H, DEP=D, deltaX=2 * math.pi / L, deltaY=math.pi / H, deltaZ=math.pi / D,
                deltaT=1e-5, Answer=0, numstep=0, mu_L=dU * 1.0 / Re, Pr_L=0.72, Pr_T=0.8, Cs=0.01,
                BL_HIG=0, Ua=0.0, Va=0.0, Wa=0.0, Ns_min=10, Nst=50, f_step=50, nStages=3,
                maxCoNum=0.5, setup=1, cfl_mode=1, seed_X=0.317391239817, precision=precision,
                sgs=sgs, recon=recon), dU


def run_arm(fsl, cfg, arm, steps, every, seed):
    name, prec, sgs, recon = arm
    L, H, D = cfg["grid"]
    p, dU = params(cfg["grid"], cfg["Mc"], cfg["Re"], prec, sgs, recon)
    state, _ = fsl.temporal_state(p, cfg["Mc"], 1.0, 1e-3, seed)
    d = fsl.Domain(p)
    d.upload_state(state)
    if sgs == 1:
        d.closure_set_scales(1.0 / dU, 1.0)
        d.closure_set_weights(fsl.closure_weights())
    dy = math.pi / H
    hist = [(0, fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)["theta"])]
    t0 = time.time()
    done = 0
    while done < steps:
        n = min(every, steps - done)
        d.step(n)
        done += n
        d.sync()
        hist.append((done, fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)["theta"]))
    wall = time.time() - t0
    stats = fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)
    u = d.download_state().reshape(L, H, 5, D).transpose(2, 0, 1, 3).copy()
    info = d.info()
    out = {"arm": name, "steps": steps, "wall_s": wall, "time": None, "theta": hist,
           "final_dt": info.deltaT}
    if sgs == 1:
        st = d.closure_stats()
        out["closure"] = {"judgements": st.judgements, "fallbacks": st.fallbacks,
                          "using_dynamic": st.using_dynamic, "visc_err": st.visc_err}
    d.close()
    return out, u, stats


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=sorted(CONFIGS) + ["turb"], default="c2")
    ap.add_argument("--steps", type=int, default=0, help="0: the configuration's own step count")
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--seed", type=int, default=20251203)
    ap.add_argument("--arms", default="", help="comma-separated subset of the configuration's arms")
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(HERE))
    import freeshearlayer_b200 as fsl

    if args.config == "turb":
        # the SGS models in a layer that turns turbulent (closure_gain)
        from freeshearlayer_b200 import closure_gain
        out = closure_gain.run(fsl, grid=(256, 128, 128), Mc=0.6, Re=2e4, amp=0.05,
                               steps=args.steps or 20000, every=args.every * 5, seed=args.seed)
        print(json.dumps(out), flush=True)
        return
    cfg = CONFIGS[args.config]
    steps = args.steps or cfg["steps"]
    want = set(a for a in args.arms.split(",") if a)
    results = {}
    for arm in cfg["arms"]:
        if want and arm[0] not in want:
            continue
        out, u, stats = run_arm(fsl, cfg, arm, steps, args.every, args.seed)
        print(json.dumps(out), flush=True)
        results[arm[0]] = (out, u, stats)
    first = next(iter(results.values()))[0]
    summary = {"config": args.config, "grid": list(cfg["grid"]), "Mc": cfg["Mc"], "Re": cfg["Re"], "steps": steps,
               "theta0": first["theta"][0][1], "arms": {}}
    for name, against in cfg["pairs"]:
        if name not in results or against not in results:
            continue
        ref_out, ref_u, ref_stats = results[against]
        out, u, stats = results[name]
        g_ref = ref_out["theta"][-1][1] - ref_out["theta"][0][1]
        mom = float(np.sqrt(sum(np.linalg.norm(ref_u[v]) ** 2 for v in (1, 2, 3))))
        g = out["theta"][-1][1] - out["theta"][0][1]
        rel = {n: float(np.linalg.norm(u[v] - ref_u[v]) / np.linalg.norm(ref_u[v]))
               for n, v in (("rho", 0), ("rho_u", 1), ("rho_v", 2), ("rho_w", 3), ("E", 4))}
        mrel = {n: float(np.linalg.norm(u[v] - ref_u[v]) / mom) for n, v in (("rho_u", 1), ("rho_v", 2), ("rho_w", 3))}
        rs = {}
        for comp in ("R11", "R22", "R33", "R12"):
            den = float(np.max(np.abs(ref_stats[comp])))
            rs[comp] = float(np.max(np.abs(stats[comp] - ref_stats[comp])) / den) if den > 0 else None
        th = np.array([t for _, t in out["theta"]]) - np.array([t for _, t in ref_out["theta"]])
        summary["arms"][name + " vs " + against] = {
            "rel_l2": rel, "momentum_l2_over_momentum_norm": mrel, "theta_growth": g, "theta_growth_against": g_ref,
            "theta_growth_rel_diff": (g - g_ref) / g_ref if g_ref else None,
            "theta_history_max_abs_diff": float(np.max(np.abs(th))),
            "reynolds_stress_max_rel_diff": rs, "wall_s": out["wall_s"], "wall_s_against": ref_out["wall_s"],
            "closure": out.get("closure")}
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
