"""Shared test helpers: parameter sets, seeded states and comparisons."""
from __future__ import annotations

import math

import numpy as np


def spatial_params(L=12, H=8, D=6, **kw) -> dict:
    """The reference's shipped layer2.ini physics on a small grid, RK3."""
    p = dict(LEN=L, HIG=H, DEP=D, deltaX=1.6666667, deltaY=1.0, deltaZ=1.5,
             deltaT=0.0007, Answer=0, numstep=10, mu_L=0.253358, Pr_L=0.72, Pr_T=0.8,
             Cs=0.01, BL_HIG=2, Ua=35.0, Va=35.0, Wa=35.0, Ns_min=10, Nst=50,
             f_step=50, nStages=3, maxCoNum=0.1, setup=0, cfl_mode=0,
             seed_X=0.317391239817)
    p.update(kw)
    return p


def temporal_params(L=16, H=8, D=8, Mc=0.4, Re=500.0, **kw) -> dict:
    """Temporal shear layer on a 2pi x pi x pi box scaled to L x H x D cells
    (dx = dy = dz), acoustic CFL 0.5, RK3; mu_L from Re = dU delta_w0 / nu."""
    dx = 2 * math.pi / L
    dU = 2.0 * Mc * math.sqrt(1.4 * 1e5 / 1.0)
    p = dict(LEN=L, HIG=H, DEP=D, deltaX=dx, deltaY=dx, deltaZ=dx, deltaT=1e-4,
             Answer=0, numstep=10, mu_L=1.0 * dU * 1.0 / Re, Pr_L=0.72, Pr_T=0.8,
             Cs=0.01, BL_HIG=0, Ua=0.0, Va=0.0, Wa=0.0, Ns_min=10, Nst=50,
             f_step=50, nStages=3, maxCoNum=0.5, setup=1, cfl_mode=1, seed_X=0.317391239817)
    p.update(kw)
    return p


def random_state(p: dict, seed: int = 1) -> np.ndarray:
    """A seeded, physically valid, non-smooth interior state (backup.dat layout)."""
    rng = np.random.default_rng(seed)
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    r = 1.0 + 0.2 * rng.random((L, H, D))
    u = 120.0 + 80.0 * rng.standard_normal((L, H, D))
    v = 20.0 * rng.standard_normal((L, H, D))
    w = 20.0 * rng.standard_normal((L, H, D))
    pr = 1e5 * (1.0 + 0.1 * rng.random((L, H, D)))
    s = np.empty((L, H, 5, D))
    s[:, :, 0] = r
    s[:, :, 1] = r * u
    s[:, :, 2] = r * v
    s[:, :, 3] = r * w
    s[:, :, 4] = pr / 0.4 + 0.5 * r * (u * u + v * v + w * w)
    return s.ravel()


def max_ulp(a: np.ndarray, b: np.ndarray) -> int:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    ia = np.where(ia < 0, np.int64(-0x8000000000000000) - ia, ia)
    ib = np.where(ib < 0, np.int64(-0x8000000000000000) - ib, ib)
    return int(np.max(np.abs(ia - ib))) if a.size else 0


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def per_var_rel_l2(sa: np.ndarray, sb: np.ndarray, p: dict):
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    a = np.asarray(sa).reshape(L, H, 5, D)
    b = np.asarray(sb).reshape(L, H, 5, D)
    return [rel_l2(a[:, :, v], b[:, :, v]) for v in range(5)]
