"""Ensembles: graph-replayed steps of independent shear layers give the same
bits as stepping each member alone; the autotuner changes no result."""
import math

import numpy as np
import pytest

from tests.helpers import temporal_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


# uneven grids, Mach and Reynolds numbers, precisions, closures and
# reconstructions
MEMBERS = [
    dict(L=24, H=16, D=16, Mc=0.3, Re=400.0, precision=0, sgs=0, seed=1),
    dict(L=32, H=12, D=24, Mc=0.5, Re=700.0, precision=1, sgs=0, seed=2),
    dict(L=16, H=24, D=12, Mc=0.7, Re=1000.0, precision=1, sgs=1, seed=3),
    dict(L=40, H=16, D=8, Mc=0.2, Re=300.0, precision=0, sgs=1, seed=4),
    dict(L=24, H=20, D=36, Mc=0.6, Re=550.0, precision=1, sgs=0, seed=5),
    dict(L=20, H=16, D=20, Mc=0.5, Re=600.0, precision=1, sgs=1, seed=6, recon=1),
    dict(L=28, H=12, D=16, Mc=0.4, Re=450.0, precision=0, sgs=0, seed=7, recon=1),
]


def _member(fsl, m, amp=1e-2):
    p = temporal_params(L=m["L"], H=m["H"], D=m["D"], Mc=m["Mc"], Re=m["Re"], precision=m["precision"],
                        sgs=m["sgs"], recon=m.get("recon", 0))
    s, dU = fsl.temporal_state(p, m["Mc"], 1.0, amp, m["seed"])
    d = fsl.Domain(p)
    d.upload_state(s)
    if m["sgs"] == 1:
        d.closure_set_scales(1.0 / dU, 1.0)
        d.closure_set_weights(fsl.closure_weights())
        d.closure_judge(0, 1.0)
    return d


def test_ensemble_matches_members_stepped_alone(fsl):
    ens_m = [_member(fsl, m) for m in MEMBERS]
    ref_m = [_member(fsl, m) for m in MEMBERS]
    e = fsl.Ensemble(ens_m)
    e.set_chunk(5)
    e.step(23)  # one plain warm-up step, 4 replays of 5, a 2-step tail graph
    e.step(10)  # 2 replays of the cached graph
    e.sync()
    for d, r in zip(ens_m, ref_m):
        r.step(33)
        a, b = d.download_state(), r.download_state()
        assert np.all(np.isfinite(a))
        assert np.array_equal(a, b)
        ia, ib = d.info(), r.info()
        assert ia.step == ib.step == 33 and ia.deltaT == ib.deltaT
    e.close()


def test_tuner_changes_no_result(fsl):
    """The tuner restores every member; with the tile shape it chose, the
    ensemble still matches members stepped alone.  (The FP32-bulk kernels'
    last bits may depend on the tile shape: the compiler may contract a face
    flux into FMAs differently where a block's march starts.)"""
    ens_m = [_member(fsl, m) for m in MEMBERS[:3] + MEMBERS[5:6]]
    ref_m = [_member(fsl, m) for m in MEMBERS[:3] + MEMBERS[5:6]]
    e = fsl.Ensemble(ens_m)
    e.step(4)
    rows, seg, ms = e.tune(trial_steps=2)
    assert rows in (0, 8, 12, 16) and seg in (8, 16, 32, 48, 64) and ms > 0
    e.step(6)
    e.sync()
    for d, r in zip(ens_m, ref_m):
        r.step(4)
        r.tune(r.TUNE_STAGE_ROWS, rows)
        r.tune(r.TUNE_STAGE_SEG, seg)
        r.step(6)
        assert np.array_equal(d.download_state(), r.download_state())
        assert d.info().step == 10
    e.close()


def test_fp64_results_do_not_depend_on_tile_shape(fsl):
    m = dict(MEMBERS[0])
    a, b = _member(fsl, m), _member(fsl, m)
    b.tune(b.TUNE_STAGE_ROWS, 8)
    b.tune(b.TUNE_STAGE_SEG, 5)
    a.step(6)
    b.step(6)
    assert np.array_equal(a.download_state(), b.download_state())


def test_unsupported_members_are_refused(fsl):
    from tests.helpers import spatial_params
    d = fsl.Domain(spatial_params(L=12, H=8, D=6))
    e = fsl.Ensemble([d])
    with pytest.raises(fsl.FslError) as ex:
        e.step(1)
    assert ex.value.code == -7
    e.close()
    m = dict(MEMBERS[2])
    d2 = _member(fsl, m)
    d2.closure_judge(100, 0.02)
    e2 = fsl.Ensemble([d2])
    with pytest.raises(fsl.FslError) as ex:
        e2.step(1)
    assert ex.value.code == -7
    e2.close()
    d3 = _member(fsl, dict(MEMBERS[0]))
    d3.step_stage()                 # in the middle of a step
    e3 = fsl.Ensemble([d3])
    with pytest.raises(fsl.FslError) as ex:
        e3.step(1)
    assert ex.value.code == -1
    e3.close()


# members the persistent path takes: FP32 bulk, reference reconstruction
PERSISTENT = [
    dict(L=24, H=16, D=16, Mc=0.3, Re=400.0, precision=1, sgs=0, seed=11),
    dict(L=32, H=12, D=24, Mc=0.5, Re=700.0, precision=1, sgs=0, seed=12),
    dict(L=16, H=24, D=12, Mc=0.7, Re=1000.0, precision=1, sgs=1, seed=13),
    dict(L=40, H=20, D=40, Mc=0.4, Re=500.0, precision=1, sgs=0, seed=14),
    dict(L=48, H=33, D=65, Mc=0.6, Re=800.0, precision=1, sgs=1, seed=15),
    # longer members: more blocks than tiles, heads and tails
    dict(L=128, H=20, D=40, Mc=0.5, Re=600.0, precision=1, sgs=0, seed=16),
    dict(L=256, H=16, D=32, Mc=0.4, Re=500.0, precision=1, sgs=1, seed=17),
]


@pytest.mark.parametrize("sgs", [None, 2])
def test_persistent_ensemble_matches_members_stepped_alone(fsl, sgs):
    """All members FP32 bulk with the reference reconstruction: each step is
    the members' work before their first stage and one cooperative launch of
    every member's three stages (grid barriers between them); the results
    are bit-identical to stepping each member alone (dynamic procedure and
    learned closure members, or all with the static model)."""
    ms = [dict(m, sgs=sgs) if sgs is not None else m for m in PERSISTENT]
    ens_m = [_member(fsl, m) for m in ms]
    ref_m = [_member(fsl, m) for m in ms]
    e = fsl.Ensemble(ens_m)
    e.set_chunk(4)
    e.step(11)
    e.sync()
    assert e.persistent() == 1
    e.step(6)
    e.sync()
    for d, r in zip(ens_m, ref_m):
        r.step(17)
        a, b = d.download_state(), r.download_state()
        assert np.all(np.isfinite(a))
        assert np.array_equal(a, b)
        assert d.info().step == 17 and d.info().deltaT == r.info().deltaT
    e.close()


def test_persistent_ensemble_barrier_gives_up(fsl):
    """A grid barrier whose wait limit runs out ends the launch with an error
    the host reads (FSL_ERR_TIMEOUT from the sync), never a fault or a hang;
    with the states uploaded again and the limit restored, the ensemble steps
    exactly as the members do alone."""
    ms = PERSISTENT[:3]
    ens_m = [_member(fsl, m) for m in ms]
    ref_m = [_member(fsl, m) for m in ms]
    e = fsl.Ensemble(ens_m)
    e.step(2)
    e.sync()
    assert e.persistent() == 1
    e.set_barrier_limit(0)
    e.step(3)
    with pytest.raises(fsl.FslError) as ex:
        e.sync()
    assert ex.value.code == -5
    e.set_barrier_limit(1 << 24)
    for d, m in zip(ens_m, ms):
        fresh = _member(fsl, m)
        d.upload_state(fresh.download_state())
        d.set_time(0, fresh.info().deltaT)
        fresh.close()
    e.step(5)
    e.sync()
    for d, r in zip(ens_m, ref_m):
        r.step(5)
        assert np.array_equal(d.download_state(), r.download_state())
    e.close()
