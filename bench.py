#!/usr/bin/env python3
"""Benchmark: cell-stage-updates/s of the explicit RK3 step on B200.

Workload (default): temporal compressible shear layer, 512 x 256 x 256 cells
(33.5 M cells, 5 conserved variables), box 2pi x pi x pi, convective Mach
0.7, Re_dw0 = 1000, acoustic CFL 0.5, RK3, dynamic Smagorinsky.  Synthetic
data: the seeded tanh profile + Crocco-Busemann temperature + uniform
velocity noise of amplitude 1e-3 dU (splitmix64 seed 20251203).

One step = one full RK3 step (Courant rescale, disturbance draw, three stages,
SGS viscosity once per step).  value = cells * 3 * steps / device seconds,
max over ranks, summed over replicas (one independent domain per GPU).

The headline arm (--arm fp32-learned) is the FP32-bulk step with the learned
closure (weights shipped in freeshearlayer_b200/closure_weights.f32) and the
dynamic procedure as judge every 100 steps.  Beside it the same box times the
plain FP64 dynamic-Smagorinsky path (plain_fp64, speedup_vs_plain_fp64) and,
from the same initial state, advances FP64, FP32 + dynamic and FP32 + learned
for --match-steps steps and reports per-variable relative L2 against FP64,
momentum-thickness growth and Reynolds-stress profile differences
(matched_error).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--arm ARM]
        (--gpus N > 1 without a launcher starts N ranks under torch.distributed.run)
    python bench.py --impl reference ...   # the reference's serial CPU solver

Prints exactly one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "cell-stage-updates/s on 1 B200: FP32+learned closure vs plain FP64, matched error"
UNIT = "cell-stage-updates/s"
GRID = (512, 256, 256)
MC, RE, DW0, AMP, SEED = 0.7, 1000.0, 1.0, 1e-3, 20251203
STAGES = 3


def workload_params(grid=GRID, precision=0, sgs=0, recon=0):
    L, H, D = grid
    dx = 2 * math.pi / L
    dU = 2.0 * MC * math.sqrt(1.4 * 1e5 / 1.0)
    return dict(LEN=L, HIG=H, DEP=D, deltaX=dx, deltaY=math.pi / H, deltaZ=math.pi / D,
                deltaT=1e-5, Answer=0, numstep=0, mu_L=1.0 * dU * DW0 / RE, Pr_L=0.72,
                Pr_T=0.8, Cs=0.01, BL_HIG=0, Ua=0.0, Va=0.0, Wa=0.0, Ns_min=10, Nst=50,
                f_step=50, nStages=3, maxCoNum=0.5, setup=1, cfl_mode=1,
                seed_X=0.317391239817, precision=precision, sgs=sgs, recon=recon)


def workload_name(grid):
    return ("temporal shear layer %dx%dx%d, Mc %.1f, Re_dw0 %.0f, RK3, acoustic CFL 0.5"
            % (grid[0], grid[1], grid[2], MC, RE))


# ---------------------------------------------------------------------------
# CPU: the reference's own serial solver (oracle/_ref), one process per core
# ---------------------------------------------------------------------------
REF_SLAB = (4, 256, 256)  # per-process slab of the workload's cross-section


def _ref_worker_main(nsteps: int, nwarm: int, slab, out_path: str):
    """Runs in its own process: the reference's serial solver (FP64,
    zero-fill patch) on one slab, timing each step; writes JSON to out_path."""
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # the reference prints every step
    from oracle.oracle import RefOracle, spatial_initial_state
    L, H, D = slab
    p = dict(LEN=L, HIG=H, DEP=D, deltaX=1.6666667, deltaY=1.0, deltaZ=1.5, deltaT=0.0007,
             Answer=0, numstep=nsteps + nwarm, mu_L=0.253358, Pr_L=0.72, Pr_T=0.8, Cs=0.01,
             BL_HIG=5, Ua=35.0, Va=35.0, Wa=35.0, Ns_min=10, Nst=50, f_step=50, nStages=3,
             maxCoNum=0.1, setup=0, cfl_mode=0, seed_X=0.317391239817)
    r = RefOracle(p)
    r.set_state(spatial_initial_state(p))
    for _ in range(nwarm):
        r.step(1)
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        r.step(1)
        times.append(time.perf_counter() - t0)
    with open(out_path, "w") as f:
        json.dump({"times": times, "cells": L * H * D}, f)


def run_reference_cpu(nproc: int, nsteps: int, nwarm: int, slab=REF_SLAB):
    """nproc concurrent reference processes; returns (value, seconds, detail)."""
    import tempfile
    from oracle import oracle as orc
    if not orc.ref_available():
        orc.build(ref=True)
    if not orc.ref_available():
        return None
    tmp = tempfile.mkdtemp(prefix="fslref_")
    procs = []
    for q in range(nproc):
        out = os.path.join(tmp, "w%d.json" % q)
        cmd = [sys.executable, os.path.abspath(__file__), "--ref-worker", str(nsteps), str(nwarm),
               "%d,%d,%d" % slab, out]
        procs.append((subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE), out))
    res = []
    for pr, out in procs:
        _, err = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError("reference worker failed: %s" % err.decode()[-500:])
        with open(out) as f:
            res.append(json.load(f))
    wall = max(sum(r["times"]) for r in res)
    units = sum(r["cells"] * STAGES * len(r["times"]) for r in res)
    per_step = [max(r["times"][s] for r in res) for s in range(nsteps)]
    return units / wall, wall, per_step


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_id: str):
        self.dev = dev_id
        self.lines = []
        self.p = None

    def start(self):
        try:
            cmd = ["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits", "-lms", "200"]
            if self.dev:
                cmd += ["-i", self.dev]
            self.p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def cpu_ranges(cpus) -> str:
    """'0-55,112-167' for a sorted CPU list."""
    out, start, prev = [], None, None
    for c in cpus:
        if start is None:
            start = prev = c
        elif c == prev + 1:
            prev = c
        else:
            out.append("%d-%d" % (start, prev) if prev > start else str(start))
            start = prev = c
    if start is not None:
        out.append("%d-%d" % (start, prev) if prev > start else str(start))
    return ",".join(out)


def gpu_local_cpus(dev_uuid: str):
    """The host CPUs on the NUMA node of the GPU's PCIe root (NVML's CPU
    affinity of the device), restricted to the CPUs this process may use;
    None when NVML cannot say."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID(dev_uuid)
            ncpu = os.cpu_count() or 1
            words = pynvml.nvmlDeviceGetCpuAffinity(h, (ncpu + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * w + b for w, m in enumerate(words) for b in range(64) if (int(m) >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return sorted(cpus) or None
    except Exception:
        return None


def bind_near_gpu(dev_uuid: str):
    """Run this process on the GPU's local CPUs, so that the pinned host
    buffers of the end-to-end leg are allocated on the NUMA node whose PCIe
    root the GPU sits under (host<->device copies from the other socket's
    memory cross the inter-socket link).  Returns the CPU list, or None."""
    cpus = gpu_local_cpus(dev_uuid)
    if cpus:
        try:
            os.sched_setaffinity(0, cpus)
        except OSError:
            return None
    return cpus


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------
ARMS = {"fp32-learned": (1, 1), "fp32-dynamic": (1, 0), "fp64-dynamic": (0, 0), "fp64-learned": (0, 1)}
ARM_NAMES = {"fp32-learned": "FP32 bulk (FP64 RK accumulation), learned closure judged by the dynamic "
                             "procedure every 100 steps",
             "fp32-dynamic": "FP32 bulk (FP64 RK accumulation), dynamic Smagorinsky",
             "fp64-dynamic": "plain FP64, dynamic Smagorinsky",
             "fp64-learned": "FP64, learned closure judged by the dynamic procedure every 100 steps"}
# Algorithmic HBM bytes per cell of one fused stage launch (each array read or
# written once, halo re-reads not counted), averaged over the three RK3 stages:
#   FP64:  stage 1 reads U^n 40 + mu 8, writes 40 (88 B); stages 2, 3 read
#          U^(s) 40 + U^n 40 + mu 8, write 40 (128 B each)   -> 114.67 B
#   FP32 bulk with FP64 stage buffers: mu is FP32 (4 B)    -> 110.67 B
STAGE_BYTES = {0: (88.0 + 128.0 + 128.0) / 3.0, 1: (84.0 + 124.0 + 124.0) / 3.0}
# Arithmetic of one cell-stage as the fused stage kernel evaluates it (per
# precision: the FP32 bulk regroups the sweeps), counted exactly by
# instantiating the step's arithmetic templates with a counting number type
# (freeshearlayer_b200/csrc/flopcount.cu, built as
# freeshearlayer_b200/_build/flopcount: "fused" and "fused_fp32"; the CPU
# tests check these numbers against it).  flops = add + mul + div + sqrt.
STAGE_OPS = {0: {"add": 520, "mul": 539, "div": 53, "sqrt": 8, "cmp": 132},
             1: {"add": 481, "mul": 515, "div": 53, "sqrt": 8, "cmp": 57}}
STAGE_FLOPS = {p: o["add"] + o["mul"] + o["div"] + o["sqrt"] for p, o in STAGE_OPS.items()}
SMS = 148


def make_domain(fsl, grid, arm, state, dU, rows=0, seg=0, recon=0, poly=-1):
    prec, sgs = ARMS[arm]
    d = fsl.Domain(workload_params(grid, precision=prec, sgs=sgs, recon=recon))
    if rows:
        d.tune(d.TUNE_STAGE_ROWS, rows)
    if seg:
        d.tune(d.TUNE_STAGE_SEG, seg)
    if poly >= 0:
        d.tune(d.TUNE_CLOSURE_POLY, poly)
    d.upload_state(state)
    if sgs == 1:
        d.closure_set_scales(DW0 / dU, DW0)
        d.closure_set_weights(fsl.closure_weights())
    return d


def time_steps(torch, d, run, steps, barrier, clocks=None):
    """K steps bracketed by barrier + synchronize; CUDA events on the domain's stream."""
    ext = torch.cuda.ExternalStream(d.stream)
    d.profile(True)
    barrier()
    torch.cuda.synchronize()
    d.sync()
    if clocks:
        clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    run(steps)
    e1.record(ext)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop() if clocks else None
    kt = d.profile_read()
    d.profile(False)
    d.sync()  # raises on a non-finite state
    return ms, kt, clk


def profiled_traffic(prec):
    """DRAM bytes per cell of one stage-2 launch of the fused stage kernel
    (FP64: the ring tile; FP32 bulk: the full-lane tile), from the committed
    ncu summary: the full-size 512x256x256 capture when it has one (the line
    'full size: ... per cell X B'), else the 256x128x128 capture ('derived:
    ... per cell X B'). Returns (bytes per cell, which capture) or (None, None)."""
    import re
    name = "k_stage_fp64_256x128x128.txt" if prec == 0 else "k_wide_fp32_256x128x128.txt"
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            txt = f.read()
    except OSError:
        return None, None
    m = re.search(r"full size: .*per cell ([0-9.]+) B", txt)
    if m:
        return float(m.group(1)), "512x256x256"
    m = re.search(r"derived: .*per cell ([0-9.]+) B", txt)
    return (float(m.group(1)), "256x128x128") if m else (None, None)


def stage_roofline(kt, names, ncell, prec, peaks, traffic):
    kms = {names[i]: kt.ms[i] for i in range(8)}
    kl = {names[i]: int(kt.launches[i]) for i in range(8)}
    launches = max(kl["stage"], 1)
    alg = STAGE_BYTES[prec] * ncell
    avg_ms = kms["stage"] / launches
    achieved = alg / (avg_ms / 1e3) / 1e9
    note = None
    if traffic is None:
        per_cell, where = profiled_traffic(prec)
        if per_cell is not None:
            traffic = per_cell * ncell
            note = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one stage-2 launch at %s "
                    "(%.2f B/cell; that stage's algorithmic bytes are %d B/cell), scaled by cells"
                    % (where, per_cell, 128 if prec == 0 else 124))
    kernel = ("k_stage<double> (ring tile: fused reconstruction + Riemann + viscous flux + divergence + RK stage)"
              if prec == 0 else
              "k_wide (FP32 full-lane persistent tile: fused reconstruction + Riemann + viscous flux + divergence "
              "+ RK stage)")
    return {"bound": "hbm", "kernel": kernel,
            "achieved": round(achieved, 2), "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic, "traffic_note": note,
            "peak_source": peaks["source"] + " HBM copy bandwidth (burst)",
            "alg_bytes_per_cell": round(STAGE_BYTES[prec], 2), "alg_bytes_per_launch": alg,
            "avg_launch_ms": round(avg_ms, 4), "launches": launches}, kms, kl


def compute_roof(roof, prec, clk):
    """The stage kernel's arithmetic rate against the vector (non-tensor) peak
    of its precision: 148 SMs x 128 FP32 (64 FP64) lanes x 2 flops (an FMA)
    per cycle at the median SM clock sampled during the timed region."""
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    lanes = 64 if prec == 0 else 128
    peak = SMS * lanes * 2 * mhz * 1e6 / 1e12
    cells = roof["alg_bytes_per_launch"] / roof["alg_bytes_per_cell"]
    achieved = STAGE_FLOPS[prec] * cells / (roof["avg_launch_ms"] / 1e3) / 1e12
    return {"bound": "fp64 vector" if prec == 0 else "fp32 vector", "flops_per_cell_stage": STAGE_FLOPS[prec],
            "ops_per_cell_stage": STAGE_OPS[prec], "achieved": round(achieved, 3), "peak": round(peak, 2),
            "unit": "TFLOP/s", "frac": round(achieved / peak, 4), "sm_mhz": mhz,
            "note": "nominal peak counts an FMA as 2 flops; divisions and square roots count 1 flop each "
                    "but issue as several instructions" +
                    ("; the FP64 path is compiled without contraction, so each add and multiply issues "
                     "on its own (half the FMA peak is its ceiling)" if prec == 0 else "")}


# the stated accuracy bar: relative L2 of each conserved variable against the
# FP64 path, each variable against its own norm
L2_BAR = 1e-5
VAR_NAMES = ["rho", "rho_u", "rho_v", "rho_w", "E"]


def rel_l2(a, b):
    import numpy as np
    return [float(np.linalg.norm(a[v] - b[v]) / max(np.linalg.norm(b[v]), 1e-300)) for v in range(5)]


def matched_error(fsl, grid, state, dU, nsteps, rows, seg):
    """Advance the same initial state nsteps with the plain FP64 path, FP32
    bulk + dynamic and FP32 bulk + learned closure; compare the conserved
    variables, momentum thickness growth and Reynolds-stress profiles."""
    import numpy as np
    L, H, D = grid
    dy = math.pi / H
    out = {"steps": nsteps}
    res = {}
    for arm in ("fp64-dynamic", "fp32-dynamic", "fp32-learned"):
        d = make_domain(fsl, grid, arm, state, dU, rows, seg)
        s0 = fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)
        d.step(nsteps)
        d.sync()
        s1 = fsl.shear_statistics(d.plane_sums(), L * D, dU, dy)
        u = d.download_state().reshape(L, H, 5, D).transpose(2, 0, 1, 3).copy()
        cst = d.closure_stats() if ARMS[arm][1] else None
        res[arm] = (u, s0, s1, cst)
        d.close()
    ref_u, ref_s0, ref_s1, _ = res["fp64-dynamic"]
    g_ref = ref_s1["theta"] - ref_s0["theta"]
    out["theta0"] = ref_s0["theta"]
    out["theta_growth_fp64"] = g_ref
    for arm in ("fp32-dynamic", "fp32-learned"):
        u, s0, s1, cst = res[arm]
        g = s1["theta"] - s0["theta"]
        rs = {}
        for comp in ("R11", "R22", "R33", "R12"):
            den = float(np.max(np.abs(ref_s1[comp])))
            rs[comp] = float(np.max(np.abs(s1[comp] - ref_s1[comp])) / den) if den > 0 else None
        mom = float(np.sqrt(sum(np.linalg.norm(ref_u[v]) ** 2 for v in (1, 2, 3))))
        rel = dict(zip(VAR_NAMES, rel_l2(u, ref_u)))
        e = {"rel_l2_vs_fp64": rel,
             "bar": L2_BAR,
             "pass": {n: bool(x <= L2_BAR) for n, x in rel.items()},
             "all_pass": bool(all(x <= L2_BAR for x in rel.values())),
             # an extra column only: the transverse momenta over the whole
             # momentum's norm (their own norms are the velocity noise)
             "l2_vs_fp64_over_momentum_norm": {n: float(np.linalg.norm(u[v] - ref_u[v]) / mom)
                                               for n, v in (("rho_u", 1), ("rho_v", 2), ("rho_w", 3))},
             "theta_growth": g,
             "theta_growth_rel_diff": (g - g_ref) / g_ref if g_ref != 0 else None,
             "reynolds_stress_max_rel_diff": rs}
        if cst is not None:
            e["closure"] = {"judgements": int(cst.judgements), "fallbacks": int(cst.fallbacks),
                            "using_dynamic": int(cst.using_dynamic),
                            "cs2_profile_err": cst.profile_err, "mu_sgs_profile_err": cst.mu_profile_err,
                            "visc_err": cst.visc_err}
        out[arm] = e
    return out


def ensemble_members(n, seed=20251203):
    """The batched-ensemble workload: n temporal shear layers, grids drawn from
    {48,64,96,128} x {32,48,64} x {32,48,64}, Mc uniform in [0.2, 0.8],
    Re_dw0 uniform in [300, 1000], perturbation seeds 0..n-1 at 1e-3 dU,
    FP32 bulk with FP64 accumulation, dynamic Smagorinsky."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        L = int(rng.choice([48, 64, 96, 128]))
        H = int(rng.choice([32, 48, 64]))
        D = int(rng.choice([32, 48, 64]))
        Mc = float(rng.uniform(0.2, 0.8))
        Re = float(rng.uniform(300.0, 1000.0))
        dU = 2.0 * Mc * math.sqrt(1.4 * 1e5 / 1.0)
        p = dict(workload_params((L, H, D), precision=1, sgs=0), mu_L=dU * DW0 / Re)
        out.append((p, Mc, q))
    return out


def ensemble_block(fsl, torch, steps, n):
    """Aggregate cell-stage updates/s of n members advanced one after another
    (each alone, fsl_step) and as one graph-replayed ensemble, both with the
    tile shape the autotuner picks for the ensemble, from the same initial
    states; the final states must agree bitwise.  When the tuner does not pick
    the persistent path (one cooperative launch of all members' stages per
    step), that path is timed too."""
    import numpy as np
    members = ensemble_members(n)
    doms, states = [], []
    for p, Mc, sd in members:
        st, _ = fsl.temporal_state(p, Mc, DW0, AMP, sd)
        d = fsl.Domain(p)
        d.upload_state(st)
        doms.append(d)
        states.append(st)
    cells = sum(p["LEN"] * p["HIG"] * p["DEP"] for p, _, _ in members)
    units = cells * STAGES * steps
    for d in doms:
        d.step(1)  # allocation and kernel attributes outside the timed region
        d.sync()
    def reset():  # same initial state and time step for every run
        for d, st, (p, _, _) in zip(doms, states, members):
            d.upload_state(st)
            d.set_time(0, p["deltaT"])

    # the tile shape the autotuner picks for the ensemble; the members stepped
    # one after another use the same shape, so the ratio compares schedules
    e = fsl.Ensemble(doms)
    e.step(1)
    rows, seg, _ = e.tune(trial_steps=5)
    e.close()
    # members one after another
    reset()
    seq_ms = 0.0
    for d in doms:
        ext = torch.cuda.ExternalStream(d.stream)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(ext)
        d.step(steps)
        b.record(ext)
        b.synchronize()
        seq_ms += a.elapsed_time(b)
    # the ensemble, with the autotuned tile shape (the members kept it)
    e = fsl.Ensemble(doms)
    reset()
    e.step(1)  # the warm-up step after an upload runs uncaptured
    e.sync()
    ext = torch.cuda.ExternalStream(e.stream)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(ext)
    e.step(steps - 1)
    b.record(ext)
    b.synchronize()
    e.sync()
    ens_ms = a.elapsed_time(b)
    ens_final = [d.download_state() for d in doms]
    e.close()
    # members alone with the ensemble's tile shape: the same bits
    reset()
    for d in doms:
        d.step(steps)
    same = all(np.array_equal(d.download_state(), f) for d, f in zip(doms, ens_final))
    ens_units = cells * STAGES * (steps - 1)
    # the persistent path (one cooperative launch of every member's stages
    # per step) when the tuner chose another shape
    pers = None
    if rows != 0:
        reset()
        for d in doms:
            d.tune(d.TUNE_STAGE_ROWS, 0)
        e = fsl.Ensemble(doms)
        e.step(1)
        e.sync()
        if e.persistent():
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            ext = torch.cuda.ExternalStream(e.stream)
            a.record(ext)
            e.step(steps - 1)
            b.record(ext)
            b.synchronize()
            e.sync()
            pms = a.elapsed_time(b)
            pers = {"value": ens_units / (pms / 1e3), "ms": pms, "steps": steps - 1}
        e.close()
    for d in doms:
        d.close()
    return {"workload": "%d temporal shear layers, grids {48,64,96,128}x{32,48,64}x{32,48,64}, Mc U[0.2,0.8], "
                        "Re_dw0 U[300,1000], noise 1e-3 dU, FP32 bulk + FP64 accumulation, dynamic Smagorinsky"
                        % n,
            "members": n, "cells": cells, "steps": steps,
            "sequential": {"value": units / (seq_ms / 1e3), "ms": seq_ms},
            "ensemble": {"value": ens_units / (ens_ms / 1e3), "ms": ens_ms, "steps": steps - 1,
                         "tile_rows": rows, "planes_per_block": seg, "chunk": 10,
                         "persistent": rows == 0},
            "persistent_rows0": pers,
            "speedup": (ens_units / ens_ms) / (units / seq_ms), "bit_identical": bool(same)}


def slab_block(fsl, torch, grid, state, dU, steps, nslabs, warmup):
    """The FP64 domain split into x-slabs on one GPU (overlap planes through
    device buffers), with the overlap exchanged once per step and after every
    stage, against the undivided domain.  The exchanges synchronise with the
    host, so all three arms are timed by the host clock around
    torch.cuda.synchronize(); the owned planes are compared bitwise."""
    import time

    import numpy as np

    from freeshearlayer_b200.slabs import SlabSet
    p = workload_params(grid)
    ncell = grid[0] * grid[1] * grid[2]
    out = {"path": ARM_NAMES["fp64-dynamic"], "slabs": nslabs, "staging": "device", "steps": steps,
           "timing": "host clock around torch.cuda.synchronize()"}

    def timed(run):
        for _ in range(warmup):
            run(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run(steps)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3

    d = make_domain(fsl, grid, "fp64-dynamic", state, dU)
    ms = timed(d.step)
    ref = d.download_state()
    d.close()
    out["whole"] = {"ms_per_step": ms / steps, "value": ncell * STAGES * steps / (ms * 1e-3)}
    for mode in ("step", "stage"):
        with SlabSet(p, nslabs, staging="device", exchange=mode) as ss:
            ss.upload_state(state)
            ms = timed(ss.step)
            same = bool(np.array_equal(ss.download_state(), ref))
            out[mode] = {"overlap": ss.W, "ms_per_step": ms / steps,
                         "value": ncell * STAGES * steps / (ms * 1e-3), "bit_identical": same,
                         "planes_stepped": int(sum(x.local_len for x in ss.slabs))}
    return out


def max_over_ranks(torch, dist, x, device="cuda"):
    """The job's time: the maximum of x over all ranks (x itself without a
    process group)."""
    if dist is None:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_max):
    """Units all ranks processed over the slowest rank's time (weak scaling:
    every rank owns the same work)."""
    return units_per_rank * world / (ms_max / 1e3)


def main_gpu(args):
    import numpy as np
    import torch
    import freeshearlayer_b200 as fsl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def maxr(x):
        return max_over_ranks(torch, dist, x)

    grid = tuple(int(x) for x in args.grid.split("x"))
    ncell = grid[0] * grid[1] * grid[2]
    arm = args.arm
    prec = ARMS[arm][0]
    state, dU = fsl.temporal_state(workload_params(grid), MC, DW0, AMP, SEED + rank)
    peaks = measured_peaks()
    names = fsl.K_CLASSES

    dev_uuid = ""
    try:
        dev_uuid = str(torch.cuda.get_device_properties(local).uuid)
        if dev_uuid and not dev_uuid.startswith("GPU-"):
            dev_uuid = "GPU-" + dev_uuid
    except Exception:
        dev_uuid = str(local)
    near = None if args.no_numa_bind else bind_near_gpu(dev_uuid)

    # ---- the headline arm: K steps, state resident in HBM ----
    d = make_domain(fsl, grid, arm, state, dU, args.rows, args.seg, poly=args.closure_poly)
    run = d.step_phased if args.phased else d.step
    for _ in range(args.warmup):
        run(1)
    d.sync()
    ms, kt, clk = time_steps(torch, d, run, args.steps, barrier, Clocks(dev_uuid))
    ms = maxr(ms)
    value = whole_job_rate(ncell * STAGES * args.steps, world, ms)
    roof, kms, kl = stage_roofline(kt, names, ncell, prec, peaks, args.traffic)
    cst = d.closure_stats() if ARMS[arm][1] else None

    # ---- end to end through the C ABI with pinned host buffers ----
    host_in = torch.empty(state.size, dtype=torch.float64, pin_memory=True)
    host_out = torch.empty(state.size, dtype=torch.float64, pin_memory=True)
    hin = host_in.numpy()
    hout = host_out.numpy()
    hin[:] = d.download_state()
    ne = max(1, args.e2e_steps)
    ext = torch.cuda.ExternalStream(d.stream)
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(ext)
    for _ in range(ne):
        d.upload_state_async(hin)
        run(1)
        d.download_state_async(hout)
    d.transfer_wait()
    f1.record(ext)
    f1.synchronize()
    barrier()
    e2e_ms = maxr(f0.elapsed_time(f1))
    e2e = {"value": whole_job_rate(ncell * STAGES * ne, world, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": int(state.nbytes), "d2h_bytes_per_step": int(state.nbytes),
           "steps": ne, "note": "per step: fsl_upload_state_async (pinned host -> HBM), fsl_step(1), "
                                "fsl_download_state_async (HBM -> pinned host); the copies run on copy "
                                "streams of their own, overlapping the neighbouring steps; timed to "
                                "fsl_transfer_wait after the last",
           "host_cpus": ("process bound to the GPU's local CPUs %s (pinned buffers on that NUMA node)"
                         % cpu_ranges(near)) if near else "not bound"}
    d.close()

    # ---- the plain FP64 dynamic-Smagorinsky GPU path on the same box ----
    plain = None
    if arm != "fp64-dynamic" and not args.no_plain:
        dp = make_domain(fsl, grid, "fp64-dynamic", state, dU, args.rows, args.seg)
        for _ in range(args.warmup):
            dp.step(1)
        dp.sync()
        pms, pkt, _ = time_steps(torch, dp, dp.step, args.steps, barrier)
        pms = maxr(pms)
        proof, pkms, pkl = stage_roofline(pkt, names, ncell, 0, peaks, None)
        plain = {"path": ARM_NAMES["fp64-dynamic"], "value": whole_job_rate(ncell * STAGES * args.steps, world, pms),
                 "ms_per_step": pms / args.steps, "kernels_ms": {k: round(v, 3) for k, v in pkms.items()},
                 "roofline": proof, "compute_roof": compute_roof(proof, 0, clk)}
        dp.close()

    # ---- PPM, the configs' reconstruction as written: FP32 bulk + learned
    # closure and plain FP64 (dynamic procedure), both with PPM, same grid ----
    ppm = None
    if args.ppm_steps > 0:
        ppm = {"reconstruction": "Colella-Woodward PPM on the characteristic variables (fused stage kernel)",
               "steps": args.ppm_steps}
        for a2 in ("fp32-learned", "fp64-dynamic"):
            dq = make_domain(fsl, grid, a2, state, dU, 0, 0, recon=1)
            for _ in range(args.warmup):
                dq.step(1)
            dq.sync()
            qms, qkt, _ = time_steps(torch, dq, dq.step, args.ppm_steps, barrier)
            qms = maxr(qms)
            qkms = {names[i]: round(qkt.ms[i], 3) for i in range(8)}
            ppm[a2] = {"value": whole_job_rate(ncell * STAGES * args.ppm_steps, world, qms),
                       "ms_per_step": qms / args.ppm_steps, "kernels_ms": qkms}
            dq.close()
        ppm["speedup_fp32_learned_vs_fp64"] = ppm["fp32-learned"]["value"] / ppm["fp64-dynamic"]["value"]
        if plain is not None:
            ppm["fp32_learned_ppm_vs_plain_fp64"] = ppm["fp32-learned"]["value"] / plain["value"]

    # ---- matched error: same initial state, M steps, against the plain FP64 path ----
    match = None
    if rank == 0 and args.match_steps > 0:
        match = matched_error(fsl, grid, state, dU, args.match_steps, args.rows, args.seg)

    # ---- what the learned closure gains, in a layer that turns turbulent ----
    gain = None
    if rank == 0 and args.gain_steps > 0:
        from freeshearlayer_b200 import closure_gain
        g = tuple(int(x) for x in args.gain_grid.split("x"))
        gain = closure_gain.run(fsl, grid=g, steps=args.gain_steps, every=500)
        for e in gain["arms"].values():  # the histories stay in validate's output
            e.pop("theta_history", None)
            e.pop("r12_max_history", None)
        gain["apriori"] = gain["apriori"][-3:]

    # ---- batched ensemble of small uneven layers against the same run one by one ----
    ens = None
    if rank == 0 and args.ens_steps > 1:
        ens = ensemble_block(fsl, torch, args.ens_steps, args.ens_members)

    # ---- x-slabs on one GPU: overlap exchanged per step or per stage ----
    slabs = None
    if rank == 0 and world == 1 and args.slab_steps > 0:
        slabs = slab_block(fsl, torch, grid, state, dU, args.slab_steps, args.slabs, args.warmup)

    # ---- CPU baseline: the reference's serial solver, rank 0 at N = 1 only ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            r = run_reference_cpu(1, args.cpu_steps, 1)
            if r:
                cpu = {"value": r[0], "unit": UNIT, "cores": 1, "kind": "reference",
                       "sample": "reference serial src (FP64, zero-fill patch) on a %dx%dx%d slab of "
                                 "the workload's cross-section, %d RK3 steps after 1 warm-up"
                                 % (REF_SLAB + (args.cpu_steps,))}
        except Exception as ex:  # report, never fall back
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "error": str(ex)[:200]}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == 0 else "f32 bulk / f64 accumulation",
                "data": "synthetic (seeded tanh shear layer, Crocco-Busemann T, uniform noise 1e-3 dU)",
                "config": {"workload": workload_name(grid), "grid": list(grid), "cells": ncell,
                           "stages_per_step": STAGES,
                           "path": ("per-phase kernels, " if args.phased else "fused stage kernels, ") +
                                   ARM_NAMES[arm],
                           "l2": "inputs larger than L2 (state %.2f GB per domain)" % (state.nbytes / 1e9),
                           "parallelism": "replicas (one independent domain per GPU)"},
                "roofline": roof, "compute_roof": compute_roof(roof, prec, clk),
                "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": int(sum(kl.values())),
                "kernels_ms": {k: round(v, 3) for k, v in kms.items()},
                "clocks": clk}
        if cst is not None:
            line["closure"] = {"judgements": int(cst.judgements), "fallbacks": int(cst.fallbacks),
                               "using_dynamic": int(cst.using_dynamic), "mu_sgs_profile_err": cst.mu_profile_err,
                               "visc_err": cst.visc_err}
        if plain is not None:
            line["plain_fp64"] = plain
            line["speedup_vs_plain_fp64"] = value / plain["value"]
        if ppm is not None:
            line["ppm"] = ppm
        if match is not None:
            line["matched_error"] = match
        if gain is not None:
            line["closure_gain"] = gain
        if ens is not None:
            line["ensemble"] = ens
        if slabs is not None:
            line["slabs"] = slabs
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    grid = tuple(int(x) for x in args.grid.split("x"))
    nproc = min(host_cores(), 128)
    why = "reference oracle library (oracle/_ref) is not built and the reference sources are absent"
    try:
        r = run_reference_cpu(nproc, args.steps, args.warmup)
    except Exception as ex:
        r = None
        why = "reference run failed: " + str(ex)[:200]
    if not r:
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    value, wall, per_step = r
    sample = ("reference serial src (FP64, zero-fill patch), %d concurrent processes each on a "
              "%dx%dx%d slab of the workload's cross-section (no halo exchange: src-par needs MPI, "
              "absent), %d RK3 steps after %d warm-up" % ((nproc,) + REF_SLAB + (args.steps, args.warmup)))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * max(per_step) if per_step else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the reference's own step-profile initial state)",
            "config": {"workload": workload_name(grid), "grid": list(grid),
                       "parallelism": "%d host processes" % nproc},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def free_port() -> int:
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def launch_ranks(n: int) -> int:
    """Run this script once per GPU under torch.distributed.run (one process
    per GPU, rendezvous on 127.0.0.1), as the multi-GPU launch would; rank 0
    prints the JSON line.  Returns the launcher's exit code."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)]
    return subprocess.call(cmd + sys.argv[1:])


def main_launcher_check(args):
    """The multi-rank plumbing without any GPU work: every rank joins the
    process group (backend FSL_BENCH_BACKEND, default nccl), the per-rank
    times (10 + rank ms) are combined by the maximum over ranks, and rank 0
    prints the fields of the line that depend on the ranks."""
    import datetime
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    backend = os.environ.get("FSL_BENCH_BACKEND", "nccl")
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    ms = max_over_ranks(torch, dist, 10.0 + rank, "cpu" if backend == "gloo" else "cuda")
    if rank == 0:
        print(json.dumps({"n_gpus": world, "ms_max": ms, "value": whole_job_rate(1000, world, ms),
                          "backend": backend}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fsl", choices=["fsl", "reference"])
    ap.add_argument("--grid", default="x".join(str(x) for x in GRID))
    ap.add_argument("--arm", default="fp32-learned", choices=sorted(ARMS))
    ap.add_argument("--phased", action="store_true", help="per-phase kernels instead of the fused step")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-numa-bind", action="store_true",
                    help="leave the process on all CPUs (default: the GPU's local CPUs)")
    ap.add_argument("--rows", type=int, default=0, help="fused stage tile rows (8, 12, 16)")
    ap.add_argument("--seg", type=int, default=0, help="x planes per fused stage block")
    ap.add_argument("--closure-poly", type=int, default=-1,
                    help="closure SiLU pairs of 8 on the FMA-pipe tanh (0, 2..6; -1: the library default)")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 path beside the arm")
    ap.add_argument("--ppm-steps", type=int, default=20,
                    help="steps timed with PPM reconstruction (FP32 + closure and FP64); 0 skips them")
    ap.add_argument("--ens-steps", type=int, default=500, help="steps of the ensemble comparison (0: skip)")
    ap.add_argument("--ens-members", type=int, default=32)
    ap.add_argument("--slab-steps", type=int, default=0,
                    help="steps of the x-slab comparison on one GPU (0: skip)")
    ap.add_argument("--slabs", type=int, default=2)
    ap.add_argument("--match-steps", type=int, default=200,
                    help="steps of the matched-error comparison against the plain FP64 path (0: skip)")
    ap.add_argument("--gain-steps", type=int, default=10000,
                    help="steps of the turbulent comparison of SGS models (0: skip)")
    ap.add_argument("--gain-grid", default="128x64x64")
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per launch of the dominant kernel from an ncu capture")
    ap.add_argument("--ref-worker", nargs=4, default=None, help=argparse.SUPPRESS)
    ap.add_argument("--launcher-check", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.ref_worker:
        n, w, slab, out = args.ref_worker
        _ref_worker_main(int(n), int(w), tuple(int(x) for x in slab.split(",")), out)
        return
    # one process per GPU: without a launcher's WORLD_SIZE, --gpus N > 1
    # starts the N ranks itself; under a launcher the two must agree
    world_env = os.environ.get("WORLD_SIZE")
    if world_env is None and args.gpus > 1:
        sys.exit(launch_ranks(args.gpus))
    if world_env is not None and int(world_env) != args.gpus:
        sys.exit("bench.py: --gpus %d, but the launcher started %s ranks (WORLD_SIZE)" % (args.gpus, world_env))
    if args.launcher_check:
        main_launcher_check(args)
        return
    if args.warmup < 3 and args.impl == "fsl":
        args.warmup = 3
    if args.impl == "reference":
        main_reference(args)
    else:
        main_gpu(args)


if __name__ == "__main__":
    main()
