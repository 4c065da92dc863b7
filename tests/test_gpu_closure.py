"""The learned closure: tensor-core forward/backward against the CPU oracle,
GPU-harvested features against the oracle's features, training, and the
judge/fallback logic of the step."""
import math

import numpy as np
import pytest

from tests.helpers import temporal_params

pytestmark = pytest.mark.gpu

GROUPS = {"W1": (0, 1024), "b1": (1024, 1088), "W2": (1088, 5184), "b2": (5184, 5248),
          "W3": (5248, 9344), "b3": (9344, 9408), "w4": (9408, 9472), "b4": (9472, 9473)}


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


def _scales(p):
    dU = 2.0 * 0.4 * math.sqrt(1.4e5)
    return 1.0 / dU, 1.0


def _random_samples(n, seed):
    rng = np.random.default_rng(seed)
    X = np.empty((n, 8), np.float32)
    X[:, 0] = rng.uniform(0, 3, n)
    X[:, 1:6] = rng.uniform(-0.7, 0.7, (n, 5))
    X[:, 6] = rng.uniform(0.9, 1.1, n)
    X[:, 7] = 0.05
    Y = rng.uniform(0, 0.15, n).astype(np.float32)
    return X, Y


@pytest.mark.parametrize("n,mode", [(1024, 0), (1000, 0), (1024, 1)])
def test_gradient_matches_cpu_oracle(fsl, n, mode):
    from oracle import mlp_oracle as mo
    tr = fsl.Trainer(4096, seed=7)
    X, Y = _random_samples(n, 11)
    tr.set_samples(X, Y)
    tr.set_loss(mode)
    p = tr.weights()
    p[9472] = 0.05  # output bias near the targets
    tr.set_weights(p)
    g, loss = tr.gradient(n)
    wts = None
    if mode == 1:
        st = np.expm1(X[:, 0].astype(np.float64)) * X[:, 6]
        wts = mo.sample_weights(X, 1.0 / np.mean(st * st))
    loss_ref, g_ref = mo.loss_and_grad(p, X, Y, wts)
    assert abs(loss - loss_ref) / loss_ref < 2e-3, (loss, loss_ref)
    for name, (a, b) in GROUPS.items():
        ref = g_ref[a:b]
        err = np.linalg.norm(g[a:b] - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 3e-2, (name, err)


def test_features_and_forward_match_oracle(fsl):
    from oracle import mlp_oracle as mo
    from oracle.oracle import Oracle
    p = temporal_params(L=24, H=12, D=16)
    s, dU = Oracle.temporal_state(p, 0.4)
    d = fsl.Domain(p)
    d.upload_state(s)
    t_ref, len_ref = 1.0 / dU, 1.0
    d.closure_set_scales(t_ref, len_ref)
    tr = fsl.Trainer(p["LEN"] * p["HIG"] * p["DEP"], seed=3)
    tr.harvest(d, stride=1)
    X, Y = tr.samples()
    bL, bH, bD = p["LEN"] - 4, p["HIG"] - 4, p["DEP"] - 4
    assert len(X) == bL * bH * bD and np.all(np.isfinite(X)) and np.all(Y >= 0)
    Upad = np.stack([d.cells(0, v) for v in range(5)])
    rng = np.random.default_rng(0)
    for cell in rng.integers(0, len(X), 40):
        k = cell % bD + 3
        j = (cell // bD) % bH + 3
        i = cell // (bD * bH) + 3
        f, _ = mo.features(Upad, i, j, k, p["deltaX"], p["deltaY"], p["deltaZ"], t_ref, len_ref)
        np.testing.assert_allclose(X[cell], f, rtol=2e-5, atol=2e-6)
    params = tr.weights()
    params[9472] = 0.05
    d.closure_set_weights(params)
    ref = mo.cs2(params, X)
    # every split of the SiLU tanh between the MUFU and the FMA-pipe polynomial
    for poly in (0, 2, 3, 4, 5, 6):
        d.tune(d.TUNE_CLOSURE_POLY, poly)
        _, cs2_mlp, cs2_dyn = d.closure_compare(fields=True)
        got = cs2_mlp[3:-3, 3:-3, 3:-3].ravel()
        assert np.max(np.abs(got - ref)) < 2e-3, poly
    dyn = cs2_dyn[3:-3, 3:-3, 3:-3].ravel()
    np.testing.assert_allclose(dyn, Y, rtol=0, atol=0)


@pytest.fixture(scope="module")
def trained(fsl):
    """A closure trained on a small temporal run (FP64 dynamic procedure)."""
    p = temporal_params(L=48, H=32, D=32, Mc=0.5)
    from oracle.oracle import Oracle
    s, dU = Oracle.temporal_state(p, 0.5, amp=0.05)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.closure_set_scales(1.0 / dU, 1.0)
    tr = fsl.Trainer(1 << 20, seed=5)
    for _ in range(6):
        d.step(5)
        tr.harvest(d, stride=2)
    X, Y = tr.samples()
    var = float(np.var(Y.astype(np.float64)))
    p0 = tr.weights()
    p0[9472] = float(np.mean(Y))
    tr.set_weights(p0)
    _, loss0 = tr.gradient()
    loss = tr.train(epochs=40, batch=8192, lr=2e-3)
    w = tr.weights()
    d.closure_set_weights(w)
    st = d.closure_compare()
    return dict(p=p, dU=dU, state=d.download_state(), weights=w, var=var, loss0=loss0,
                loss=loss, n=len(Y), perr=st.profile_err, cerr=st.cell_err, merr=st.mu_profile_err,
                verr=st.visc_err)


def test_training_beats_mean_predictor(trained):
    """The per-cell dynamic coefficient is dominated by cell-to-cell noise, so
    the bar is the mean predictor (MSE = variance) per cell, and a small error
    of the plane-averaged Cs^2 profile, the quantity that sets the mean SGS
    dissipation and the judge's criterion."""
    print("samples %d var %.3e loss0 %.3e loss %.3e cs2 profile %.3f cs2 cell %.3f mu profile %.3f "
          "visc %.4f" % (trained["n"], trained["var"], trained["loss0"], trained["loss"], trained["perr"],
                         trained["cerr"], trained["merr"], trained["verr"]))
    assert trained["n"] > 50000
    assert trained["loss"] < trained["loss0"]
    assert trained["loss"] < 0.9 * trained["var"]
    assert trained["merr"] < 0.35
    assert trained["verr"] < 0.02


def test_fallback_is_the_dynamic_procedure(fsl, trained):
    """Judged every step with threshold 0, every step falls back: the run is
    bit-identical to the dynamic procedure."""
    p = dict(trained["p"])
    a = fsl.Domain(dict(p, sgs=1))
    a.upload_state(trained["state"])
    a.closure_set_scales(1.0 / trained["dU"], 1.0)
    a.closure_set_weights(trained["weights"])
    a.closure_judge(1, 0.0)
    b = fsl.Domain(p)
    b.upload_state(trained["state"])
    a.step(4)
    b.step(4)
    assert np.array_equal(a.download_state(), b.download_state())
    st = a.closure_stats()
    assert st.judgements == 4 and st.using_dynamic == 1 and st.fallbacks == 1


@pytest.mark.parametrize("prec", [0, 1])
def test_learned_closure_steps(fsl, trained, prec):
    p = dict(trained["p"], sgs=1, precision=prec)
    d = fsl.Domain(p)
    d.upload_state(trained["state"])
    d.closure_set_scales(1.0 / trained["dU"], 1.0)
    d.closure_set_weights(trained["weights"])
    d.closure_judge(5, 1e9)
    d.step(10)
    s = d.download_state()
    assert np.all(np.isfinite(s))
    st = d.closure_stats()
    assert st.judgements == 2 and st.fallbacks == 0 and st.using_dynamic == 0
    assert np.isfinite(st.mu_profile_err) and st.mu_profile_err < 0.5
    assert np.isfinite(st.visc_err) and st.visc_err < 0.05


def test_fp32_dynamic_procedure_matches_fp64(fsl, trained):
    """The FP32-bulk path's dynamic procedure (filters and coefficient in FP32)
    against the plain FP64 one on the same state: plane-averaged Cs^2 within
    1e-2 and the cell values strongly correlated."""
    out = []
    for prec in (0, 1):
        d = fsl.Domain(dict(trained["p"], sgs=1, precision=prec))
        d.upload_state(trained["state"])
        d.closure_set_scales(1.0 / trained["dU"], 1.0)
        d.closure_set_weights(trained["weights"])
        _, _, dyn = d.closure_compare(fields=True)
        out.append(dyn[3:-3, 3:-3, 3:-3].astype(np.float64))
    a64, a32 = out
    prof64, prof32 = a64.mean(axis=(0, 2)), a32.mean(axis=(0, 2))
    assert np.linalg.norm(prof32 - prof64) / np.linalg.norm(prof64) < 1e-2
    assert np.corrcoef(a64.ravel(), a32.ravel())[0, 1] > 0.99


def _active_state(fsl, oracle_lib):
    """A temporal layer whose velocity noise (5e-2 dU) at a high Reynolds
    number (2e4) makes the dynamic procedure's SGS viscosity comparable to the
    molecular one (plane averages up to several mu_L)."""
    p = temporal_params(L=48, H=32, D=32, Mc=0.5, Re=20000.0)
    s, dU = oracle_lib.Oracle.temporal_state(p, 0.5, amp=0.05)
    return p, s, dU


def _weights(fsl, kind):
    w = fsl.closure_weights().copy()
    if kind == "zero":
        return np.zeros_like(w)
    rng = np.random.default_rng(17)
    for a, b in GROUPS.values():  # every parameter group permuted within itself
        w[a:b] = rng.permutation(w[a:b])
    return w


@pytest.mark.parametrize("kind", ["zero", "shuffled"])
def test_useless_weights_fall_back(fsl, oracle_lib, kind):
    """The judge at its default thresholds catches a useless network: with the
    shipped parameters zeroed, or permuted within each layer, on a state where
    the dynamic SGS viscosity reaches more than 0.1 mu_L, the first judgement
    (step 1) falls back, and the step is then exactly the dynamic procedure's."""
    p, s, dU = _active_state(fsl, oracle_lib)
    d = fsl.Domain(dict(p, sgs=1))
    d.upload_state(s)
    d.closure_set_scales(1.0 / dU, 1.0)
    d.closure_set_weights(_weights(fsl, kind))
    d.step(1)
    st = d.closure_stats()
    print("%s: dyn_ratio %.3f active rows %d mu_active_err %.3f visc_err %.4f" %
          (kind, st.dyn_ratio, st.active_rows, st.mu_active_err, st.visc_err))
    assert st.dyn_ratio > 0.1 and st.active_rows > 0
    assert st.judgements == 1 and st.fallbacks >= 1 and st.using_dynamic == 1
    ref = fsl.Domain(p)
    ref.upload_state(s)
    ref.step(1)
    assert np.array_equal(d.download_state(), ref.download_state())


def test_shipped_weights_on_an_active_state(fsl, oracle_lib):
    """The shipped parameters judged on the same state: the errors are
    reported; both criteria are computed on the rows where the model acts."""
    p, s, dU = _active_state(fsl, oracle_lib)
    d = fsl.Domain(dict(p, sgs=1))
    d.upload_state(s)
    d.closure_set_scales(1.0 / dU, 1.0)
    d.closure_set_weights(fsl.closure_weights())
    st = d.closure_compare()
    print("shipped: dyn_ratio %.3f active rows %d mu_active_err %.3f mu_profile_err %.3f visc_err %.4f "
          "cs2_profile_err %.3f" % (st.dyn_ratio, st.active_rows, st.mu_active_err, st.mu_profile_err,
                                    st.visc_err, st.profile_err))
    assert st.active_rows > 0 and np.isfinite(st.mu_active_err)


@pytest.mark.parametrize("judge_every", [0, 3])
def test_stage_written_feature_velocities(fsl, oracle_lib, judge_every):
    """On the FP32 bulk's full-lane temporal path the last stage of a step
    writes the FP32 velocities of the new state (ghost cells included) for the
    next step's closure features, and only the first step of an fsl_step call
    runs the velocity pass. Seven steps in one call equal seven calls of one
    step (velocity pass before each) bit for bit, with and without
    judgements."""
    p, s, dU = _active_state(fsl, oracle_lib)
    out = []
    for calls in ((7,), (1,) * 7):
        d = fsl.Domain(dict(p, sgs=1, precision=1))
        d.upload_state(s)
        d.closure_set_scales(1.0 / dU, 1.0)
        d.closure_set_weights(fsl.closure_weights())
        d.closure_judge(judge_every, 1e9)
        for n in calls:
            d.step(n)
        out.append(d.download_state())
        d.close()
    assert np.array_equal(out[0], out[1])
