"""The x-reach of one RK stage and of one step, measured on the CPU oracle
by perturbing one plane with the time step held fixed: the overlap widths of
the x-slab decomposition (slabs.RADIUS for an exchange per step,
slabs.STAGE_RADIUS for an exchange per stage) must cover them.  The stage
phases run in the reference's order (src/layer2.c:163-178: ghost cells,
reconstruction, interface conditions, fluxes with the SGS viscosity of U^n,
evolution)."""
import numpy as np
import pytest

from tests.helpers import temporal_params

MID = 20


def _stage(o, s):
    o.ghost()
    o.recon()
    o.ifbc()
    o.fluxes()
    o.evolution(3, s)


def _planes(o, which, p):
    a = np.stack([o.cells(which, q)[1:-1, 1:-1, 1:-1] for q in range(5)], axis=2)
    return a.reshape(p["LEN"], -1)


def _reach(a, b):
    changed = np.nonzero(np.any(a != b, axis=1))[0] + 1
    return int(np.max(np.abs(changed - MID)))


@pytest.fixture(params=[0, 1], ids=["reference-scheme", "ppm"])
def case(request, oracle_lib):
    p = temporal_params(L=40, H=8, D=8, recon=request.param)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    return p, s


def _oracle(oracle_lib, p, s):
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.set_dt(1e-5)
    return o


def test_reach_of_one_stage(oracle_lib, case):
    from freeshearlayer_b200.slabs import STAGE_RADIUS
    p, s = case
    P = p["HIG"] * 5 * p["DEP"]
    pert = s.reshape(p["LEN"], P).copy()
    pert[MID - 1] *= 1.0 + 1e-3 * np.random.default_rng(3).random(P)
    # stage 1 from a perturbed U^n (stencil and SGS viscosity)
    out = []
    for st in (s, pert.ravel()):
        o = _oracle(oracle_lib, p, st)
        _stage(o, 1)
        out.append(_planes(o, 1, p))
    r1 = _reach(out[0], out[1])
    # stage 2 from a perturbed stage state (U^n and its SGS viscosity unchanged)
    out = []
    for perturb in (False, True):
        o = _oracle(oracle_lib, p, s)
        _stage(o, 1)
        if perturb:
            f = 1.0 + 1e-3 * np.random.default_rng(4).random((p["HIG"], p["DEP"]))
            for q in range(5):
                c = o.cells(1, q)
                c[MID, 1:-1, 1:-1] *= f
                o.set_cells(1, q, c)
        _stage(o, 2)
        out.append(_planes(o, 1, p))
    r2 = _reach(out[0], out[1])
    assert r1 == 3, r1                                # the SGS viscosity: 2, read at +-1
    assert r2 == (2 if p["recon"] == 0 else 3), r2    # the reconstruction stencil
    assert max(r1, r2) < STAGE_RADIUS[p["recon"]]     # a plane of margin


def test_reach_of_one_step(oracle_lib, case):
    from freeshearlayer_b200.slabs import RADIUS
    p, s = case
    P = p["HIG"] * 5 * p["DEP"]
    pert = s.reshape(p["LEN"], P).copy()
    pert[MID - 1] *= 1.0 + 1e-3 * np.random.default_rng(3).random(P)
    out = []
    for st in (s, pert.ravel()):
        o = _oracle(oracle_lib, p, st)
        for k in (1, 2, 3):
            _stage(o, k)
        out.append(_planes(o, 0, p))
    r = _reach(out[0], out[1])
    assert r == (7 if p["recon"] == 0 else 9), r
    assert r < RADIUS[p["recon"]]
