"""The shipped closure parameters (freeshearlayer_b200/closure_weights.f32)
on the CPU, through the MLP oracle's BF16 forward pass: the vector has the
layout the kernels read (FSL_CLOSURE_NPARAMS floats, the first layer's
padding columns zero), every value is finite, and the network answers
features of the kind it was trained on with Cs^2 that depends on them."""
import numpy as np

import freeshearlayer_b200 as fsl


def test_shipped_parameters_layout_and_response():
    from oracle import mlp_oracle as mo
    w = fsl.closure_weights()                       # checks the count
    assert w.size == fsl.CLOSURE_NPARAMS
    assert np.all(np.isfinite(w))
    assert np.all(w[:64 * 16].reshape(64, 16)[:, 8:] == 0.0)    # inputs 8..15 are padding
    rng = np.random.default_rng(1)
    n = 4096
    X = np.empty((n, 8))
    X[:, 0] = rng.uniform(0.0, 3.0, n)              # log1p(|S| t_ref)
    a = rng.normal(size=(n, 5))
    X[:, 1:6] = 0.7 * a / np.linalg.norm(a, axis=1, keepdims=True)   # strain components over |S|
    X[:, 6] = rng.uniform(0.8, 1.2, n)              # rho
    X[:, 7] = 0.05                                  # Delta / delta_w0
    y, _ = mo.forward(w.astype(np.float64), X)
    assert np.all(np.isfinite(y))
    c = mo.cs2(w.astype(np.float64), X)
    assert np.all((c >= 0.0) & (c <= 0.15))
    assert np.std(y) > 1e-4                          # not a constant predictor
