"""CPU oracle of the learned closure's MLP.  TEST INFRASTRUCTURE ONLY.

Forward and backward of the 8 -> 64 -> 64 -> 64 -> 1 SiLU network in FP64
numpy, with BF16 rounding (round to nearest even) at exactly the points where
the tensor-core kernels (freeshearlayer_b200/csrc/fsl_mlp.cu) hold BF16
operands: the features, the weights W1..W3, the hidden activations a1, a2
and the back-propagated dz of layers 3, 2, 1 that feed tensor-core products.
Pre-activations, biases, the last layer and all accumulations stay in higher
precision.  This is the training kernels' arithmetic; they evaluate sigmoid
through tanh.approx.f32, so agreement is to the few-1e-3 level, not bitwise.
The inference kernel is coarser still (its hidden SiLU runs in packed BF16 on
h = (z + b)/2 cut to BF16, biases enter the tensor-core products as BF16
high + low parts, and the output layer is a BF16 product); its tests compare
its Cs^2 with this forward pass to 2e-3 absolute.

Also: the features of one cell from the padded state, as the kernels form them.
"""
from __future__ import annotations

import numpy as np

NPARAMS = 9473
OFF = {"W1": 0, "b1": 1024, "W2": 1088, "b2": 5184, "W3": 5248, "b3": 9344, "w4": 9408, "b4": 9472}


def bf16(x: np.ndarray) -> np.ndarray:
    x32 = np.ascontiguousarray(np.asarray(x, np.float32))
    u = x32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64).reshape(np.shape(x))


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, np.float64)
    return {
        "W1": p[OFF["W1"]:OFF["b1"]].reshape(64, 16), "b1": p[OFF["b1"]:OFF["W2"]],
        "W2": p[OFF["W2"]:OFF["b2"]].reshape(64, 64), "b2": p[OFF["b2"]:OFF["W3"]],
        "W3": p[OFF["W3"]:OFF["b3"]].reshape(64, 64), "b3": p[OFF["b3"]:OFF["w4"]],
        "w4": p[OFF["w4"]:OFF["b4"]], "b4": p[OFF["b4"]],
    }


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def silu(x):
    return x * sigmoid(x)


def dsilu(x):
    s = sigmoid(x)
    return s + x * s * (1.0 - s)


def forward(p: np.ndarray, X: np.ndarray):
    w = unpack(p)
    a0 = np.zeros((len(X), 16))
    a0[:, :8] = bf16(X)
    z1 = a0 @ bf16(w["W1"]).T + w["b1"]
    a1 = bf16(silu(z1))
    z2 = a1 @ bf16(w["W2"]).T + w["b2"]
    a2 = bf16(silu(z2))
    z3 = a2 @ bf16(w["W3"]).T + w["b3"]
    a3 = silu(z3)
    y = a3 @ w["w4"] + w["b4"]
    return y, (a0, z1, a1, z2, a2, z3, a3)


def cs2(p: np.ndarray, X: np.ndarray) -> np.ndarray:
    y, _ = forward(p, X)
    return np.clip(y, 0.0, 0.15)


def sample_weights(X: np.ndarray, inv_wmean: float) -> np.ndarray:
    """(rho |S| t_ref)^2 over its mean, from the features f0 = log1p(|S| t_ref), f6 = rho."""
    X = np.asarray(X, np.float32)
    st = np.expm1(X[:, 0]).astype(np.float32) * X[:, 6]
    return (st * st * np.float32(inv_wmean)).astype(np.float64)


def loss_and_grad(p: np.ndarray, X: np.ndarray, Y: np.ndarray, weights: np.ndarray | None = None):
    """(Weighted) mean squared error of the unclipped output and its gradient (FP64)."""
    w = unpack(p)
    n = len(X)
    wt = np.ones(n) if weights is None else np.asarray(weights, np.float64)
    y, (a0, z1, a1, z2, a2, z3, a3) = forward(p, X)
    e = y - np.asarray(Y, np.float64)
    loss = float(np.mean(wt * e * e))
    dy = 2.0 * wt * e / n
    g = np.zeros(NPARAMS)
    g[OFF["w4"]:OFF["b4"]] = a3.T @ dy
    g[OFF["b4"]] = dy.sum()
    dz3 = (dy[:, None] * w["w4"][None, :]) * dsilu(z3)
    g[OFF["b3"]:OFF["w4"]] = dz3.sum(0)
    dz3b = bf16(dz3)
    g[OFF["W3"]:OFF["b3"]] = (dz3b.T @ a2).ravel()
    da2 = dz3b @ bf16(w["W3"])
    dz2 = da2 * dsilu(z2)
    g[OFF["b2"]:OFF["W3"]] = dz2.sum(0)
    dz2b = bf16(dz2)
    g[OFF["W2"]:OFF["b2"]] = (dz2b.T @ a1).ravel()
    da1 = dz2b @ bf16(w["W2"])
    dz1 = da1 * dsilu(z1)
    g[OFF["b1"]:OFF["W2"]] = dz1.sum(0)
    gW1 = bf16(dz1).T @ a0
    gW1[:, 8:] = 0.0
    g[OFF["W1"]:OFF["b1"]] = gW1.ravel()
    return loss, g


def features(Upad: np.ndarray, i: int, j: int, k: int, dx, dy, dz, t_ref: float, len_ref: float):
    """Features of padded cell (i, j, k) from the padded state Upad[5][...]
    (rho, rho u, rho v, rho w, E), in FP32 arithmetic like the kernels."""
    f32 = np.float32

    def vel(a, b, c):
        r = Upad[0, a, b, c]
        rr = f32(1.0 / r)
        return f32(Upad[1, a, b, c]) * rr, f32(Upad[2, a, b, c]) * rr, f32(Upad[3, a, b, c]) * rr

    r2x, r2y, r2z = (f32(1.0 / (4 * d) + 1.0 / (4 * d)) for d in (dx, dy, dz))
    xp, xm = vel(i + 1, j, k), vel(i - 1, j, k)
    yp, ym = vel(i, j + 1, k), vel(i, j - 1, k)
    zp, zm = vel(i, j, k + 1), vel(i, j, k - 1)
    g = np.array([[(xp[q] - xm[q]) * r2x, (yp[q] - ym[q]) * r2y, (zp[q] - zm[q]) * r2z] for q in range(3)],
                 dtype=np.float32)
    S11, S22, S33 = g[0, 0], g[1, 1], g[2, 2]
    S12 = f32(0.5) * (g[0, 1] + g[1, 0])
    S13 = f32(0.5) * (g[0, 2] + g[2, 0])
    S23 = f32(0.5) * (g[1, 2] + g[2, 1])
    S = np.sqrt(f32(2) * (S11 * S11 + S22 * S22 + S33 * S33 + f32(2) * (S12 * S12 + S13 * S13 + S23 * S23)))
    inv = f32(1) / (S + f32(1e-30))
    delta = np.cbrt(dx * dy * dz)
    return np.array([np.log1p(S * f32(t_ref)), S11 * inv, S22 * inv, S12 * inv, S13 * inv, S23 * inv,
                     f32(Upad[0, i, j, k]), f32(delta / len_ref)], np.float32), float(S)
