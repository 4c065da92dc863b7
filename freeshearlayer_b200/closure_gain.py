"""What the learned closure gains over the methods without it, in a layer
that becomes turbulent.

One temporal shear layer, seeded with strong velocity noise at a Reynolds
number high enough that the dynamic procedure's SGS viscosity reaches and
passes the molecular one once the layer has rolled up, is advanced from the
same state by five arms:

* ``fp64-dynamic``: the plain method (FP64, dynamic Smagorinsky) -- the
  reference every other arm is compared with;
* ``fp32-dynamic``: the FP32 bulk with the same model -- the precision floor
  of any comparison (in a turbulent flow two runs that differ only in
  rounding decorrelate too);
* ``fp32-learned``: the FP32 bulk with the learned closure (judged every 100
  steps, the default; while a judgement fails the steps run the dynamic
  procedure, and ``closure_steps`` counts the steps the network served);
* ``fp32-learned-only``: the network alone, judgements off;
* ``fp32-static``: the FP32 bulk with the reference's static Smagorinsky
  model (src/fluxes.c:193-205, Cs from the parameters, 0.01 as in
  layer2.ini);
* ``fp32-none``: the FP32 bulk with no SGS model.

Two kinds of error are reported against the FP64 dynamic arm:

* a priori, on the FP64 dynamic arm's own states every ``every`` steps: the
  plane-averaged SGS viscosity profile <mu>(y) of the learned closure and of
  the static model against the dynamic procedure's, all three formed from
  the same cell strain rate |S| (the dynamic procedure's central
  differences, src/turbulence.c:273-301) -- relative L2 over the rows where
  <mu_dyn> >= 0.1 mu_L (where the model acts) and over all rows;
* a posteriori, each arm's own flow: the momentum-thickness history theta(t)
  and the history of the peak Reynolds shear stress max_y |R12|(t), relative
  to the reference's growth and peak, and the final Favre Reynolds-stress
  profiles relative to their maxima.
"""
from __future__ import annotations

import math
import time

import numpy as np

ARMS = [("fp64-dynamic", 0, 0), ("fp32-dynamic", 1, 0), ("fp32-learned", 1, 1), ("fp32-learned-only", 1, 1),
        ("fp32-static", 1, 2), ("fp32-none", 1, 3)]


def layer_params(grid, Mc, Re, precision=0, sgs=0, Cs=0.01):
    L, H, D = grid
    dU = 2.0 * Mc * math.sqrt(1.4e5)
    return dict(LEN=L, HIG=H, DEP=D, deltaX=2 * math.pi / L, deltaY=math.pi / H, deltaZ=math.pi / D,
                deltaT=1e-5, Answer=0, numstep=0, mu_L=dU / Re, Pr_L=0.72, Pr_T=0.8, Cs=Cs, BL_HIG=0,
                Ua=0.0, Va=0.0, Wa=0.0, Ns_min=10, Nst=50, f_step=50, nStages=3, maxCoNum=0.5, setup=1,
                cfl_mode=1, seed_X=0.317391239817, precision=precision, sgs=sgs, recon=0), dU


def sgs_profiles(fsl, d, p, dU):
    """A-priori SGS viscosity profiles of the dynamic procedure, the learned
    closure and the static model on the domain's current U^n (band cells two
    or more from every boundary), from the same |S| and rho."""
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    _, cs2_mlp, _ = d.closure_compare(fields=True)
    tr = fsl.Trainer((L - 4) * (H - 4) * (D - 4) + 16, seed=1)
    try:
        tr.harvest(d, 1)
        X, Y = tr.samples()
    finally:
        tr.close()
    S = np.expm1(X[:, 0].astype(np.float64)) * dU  # features use t_ref = 1 / dU
    rho = X[:, 6].astype(np.float64)
    DD = (p["deltaX"] * p["deltaY"] * p["deltaZ"]) ** (2.0 / 3.0)
    shape = (L - 4, H - 4, D - 4)

    def prof(cs2):
        return (rho * cs2 * DD * S).reshape(shape).mean(axis=(0, 2))

    return (prof(Y.astype(np.float64)), prof(cs2_mlp[3:-3, 3:-3, 3:-3].ravel().astype(np.float64)),
            prof(np.full_like(S, p["Cs"])))


def _rel(a, b, mask=None):
    if mask is not None:
        if not mask.any():
            return None
        a, b = a[mask], b[mask]
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else None


def run(fsl, grid=(128, 64, 64), Mc=0.6, Re=2e4, amp=0.05, steps=10000, every=500, seed=20251203,
        weights=None, arms=None):
    """Advance the arms; returns the comparison as a dict (see the module
    docstring)."""
    L, H, D = grid
    dy = math.pi / H
    w = fsl.closure_weights(weights)
    p0, dU = layer_params(grid, Mc, Re)
    state, _ = fsl.temporal_state(p0, Mc, 1.0, amp, seed)
    out = {"workload": "temporal shear layer %dx%dx%d, Mc %.2f, Re_dw0 %.0f, noise %.2g dU, %d steps"
                       % (L, H, D, Mc, Re, amp, steps),
           "grid": list(grid), "Mc": Mc, "Re": Re, "amp": amp, "steps": steps, "every": every, "arms": {}}
    hist = {}
    apriori = []
    for name, prec, sgs in ARMS:
        if arms and name not in arms and name != "fp64-dynamic":
            continue
        p, _ = layer_params(grid, Mc, Re, prec, sgs)
        d = fsl.Domain(p)
        d.upload_state(state)
        d.closure_set_scales(1.0 / dU, 1.0)
        d.closure_set_weights(w)
        if name == "fp32-learned-only":
            d.closure_judge(0, 0.05)
        th, r12, t0 = [], [], time.time()
        done = 0
        while True:
            st = fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)
            th.append(st["theta"])
            r12.append(float(np.max(np.abs(st["R12"]))))
            if name == "fp64-dynamic":
                dyn, mlp, sta = sgs_profiles(fsl, d, p, dU)
                act = dyn >= 0.1 * p["mu_L"]
                apriori.append({"step": done, "dyn_ratio": float(np.max(dyn) / p["mu_L"]),
                                "active_rows": int(act.sum()),
                                "learned_active": _rel(mlp, dyn, act), "static_active": _rel(sta, dyn, act),
                                "learned_all": _rel(mlp, dyn), "static_all": _rel(sta, dyn)})
            if done >= steps:
                break
            n = min(every, steps - done)
            d.step(n)
            d.sync()
            done += n
        final = fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)
        info = {"wall_s": time.time() - t0, "theta": th, "r12_max": r12}
        if sgs == 1:
            cs = d.closure_stats()
            info["closure"] = {"judgements": int(cs.judgements), "fallbacks": int(cs.fallbacks),
                               "using_dynamic": int(cs.using_dynamic), "dynamic_steps": int(cs.dynamic_steps),
                               "closure_steps": steps - int(cs.dynamic_steps)}
        hist[name] = (info, final)
        d.close()
    ref, ref_final = hist["fp64-dynamic"]
    g_ref = ref["theta"][-1] - ref["theta"][0]
    r12_ref = max(ref["r12_max"])
    for name, (info, final) in hist.items():
        e = {"wall_s": info["wall_s"], "theta_growth": info["theta"][-1] - info["theta"][0],
             "theta_history": info["theta"], "r12_max_history": info["r12_max"]}
        if "closure" in info:
            e["closure"] = info["closure"]
        if name != "fp64-dynamic":
            e["theta_history_err"] = float(np.max(np.abs(np.array(info["theta"]) - np.array(ref["theta"])))
                                           / abs(g_ref)) if g_ref else None
            e["r12_history_err"] = float(np.max(np.abs(np.array(info["r12_max"]) - np.array(ref["r12_max"])))
                                         / r12_ref) if r12_ref > 0 else None
            rs = {}
            for comp in ("R11", "R22", "R33", "R12"):
                den = float(np.max(np.abs(ref_final[comp])))
                rs[comp] = float(np.max(np.abs(final[comp] - ref_final[comp])) / den) if den > 0 else None
            e["final_reynolds_stress_max_rel_diff"] = rs
        out["arms"][name] = e
    out["apriori"] = apriori

    def mean(key):
        v = [a[key] for a in apriori if a[key] is not None]
        return float(np.mean(v)) if v else None

    out["apriori_mean"] = {k: mean(k) for k in ("learned_active", "static_active", "learned_all", "static_all")}
    a = out["arms"]
    for arm in ("fp32-learned", "fp32-learned-only"):
        if arm in a and "fp32-static" in a:
            out[arm.replace("fp32-", "").replace("-", "_") + "_beats_static"] = {
                "apriori_mu_profile": (out["apriori_mean"]["learned_active"] or 1e9)
                < (out["apriori_mean"]["static_active"] or 1e9),
                "theta_history": a[arm]["theta_history_err"] < a["fp32-static"]["theta_history_err"],
                "r12_history": a[arm]["r12_history_err"] < a["fp32-static"]["r12_history_err"]}
    return out
