"""PPM reconstruction (project extension; the reference has only its
characteristic kappa = 1/3 scheme): the oracle's restatement, on the CPU.
Exact on linear data like the reference scheme, and more accurate than it on
smooth data (cell averages of a sine, edge values against the exact ones)."""
import math

import numpy as np
import pytest

from tests.helpers import temporal_params


def _sine_state(p, amp, kx):
    """Cell averages of rho = 1 + amp sin(kx x) along x; uniform u, p; v = w = 0."""
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    dx = p["deltaX"]
    xl = np.arange(L) * dx
    rho = 1.0 + amp * (np.cos(kx * xl) - np.cos(kx * (xl + dx))) / (kx * dx)
    u0, p0 = 50.0, 1e5
    s = np.empty((L, H, 5, D))
    s[:, :, 0] = rho[:, None, None]
    s[:, :, 1] = (rho * u0)[:, None, None]
    s[:, :, 2] = 0.0
    s[:, :, 3] = 0.0
    s[:, :, 4] = (p0 / 0.4 + 0.5 * rho * u0 * u0)[:, None, None]
    return s.ravel(), (xl + dx)


def _x_faces(oracle_lib, p, s):
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.ghost()
    o.recon()
    return o.faces(0, 0, 0)  # rho on the minus side of x faces (the hi state of cell i)


def _median_edge_error(oracle_lib, L, recon):
    p = temporal_params(L=L, H=6, D=6, recon=recon)
    kx = 2 * math.pi / (p["LEN"] * p["deltaX"])
    s, xface = _sine_state(p, 0.05, kx)
    f = _x_faces(oracle_lib, p, s)               # face i = right face of cell i
    exact = 1.0 + 0.05 * np.sin(kx * xface)      # right edges of cells 1..L
    return float(np.median(np.abs(f[1:, 2, 2] - exact)[2:-2]))


def test_ppm_beats_the_reference_scheme_on_smooth_data(oracle_lib):
    """Typical edge error (median over cells; both limiters clip the sine's
    extrema alike): PPM well below the reference scheme, and converging at
    fourth order (error / 16 per halving of h) against its third."""
    e = {(L, r): _median_edge_error(oracle_lib, L, r) for L in (32, 64) for r in (0, 1)}
    assert e[(32, 1)] < 0.2 * e[(32, 0)], e
    assert e[(32, 1)] / e[(64, 1)] > 12.0, e
    assert e[(32, 0)] / e[(64, 0)] < 10.0, e


def test_ppm_exact_on_constant_and_linear_data(oracle_lib):
    p = temporal_params(L=16, H=6, D=6, recon=1)
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    s = np.empty((L, H, 5, D))
    rho = 1.0 + 1e-3 * np.arange(L)  # linear, no extremum inside
    s[:, :, 0] = rho[:, None, None]
    s[:, :, 1] = 10.0 * rho[:, None, None]
    s[:, :, 2] = 0.0
    s[:, :, 3] = 0.0
    s[:, :, 4] = 1e5 / 0.4 + 0.5 * 100.0 * rho[:, None, None]
    f = _x_faces(oracle_lib, p, s.ravel())
    exact = rho + 0.5e-3                            # right face of cell i
    np.testing.assert_allclose(f[3:L - 1, 2, 2], exact[2:L - 2], rtol=0, atol=1e-12)
    q = dict(p)
    s2 = np.tile(np.array([1.2, 30.0, -4.0, 2.0, 2.6e5])[None, None, :, None], (L, H, 1, D)).ravel()
    f2 = _x_faces(oracle_lib, q, s2)
    np.testing.assert_allclose(f2[1:L, :, :], 1.2, rtol=0, atol=1e-13)
