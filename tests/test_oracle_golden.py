"""The oracle against the committed golden vectors generated from the
reference itself (tests/golden/make_golden.py).  Runs without the reference
sources: this is the pin that travels."""
import ast
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    z = np.load(os.path.join(HERE, name))
    return z, ast.literal_eval(str(z["params"][0]))


@pytest.fixture(scope="module")
def orc(oracle_lib):
    return oracle_lib


def _eq(a, b, what):
    assert np.array_equal(a, b), "%s: max |d| %g" % (what, np.max(np.abs(a - b)))


def test_golden_phases(orc):
    z, p = _load("ref_phases.npz")
    o = orc.Oracle(p)
    o.set_state(z["state_in"])
    o.set_disturbance(*[int(x) if i < 2 else float(x) for i, x in enumerate(z["disturbance"])])
    o.ghost()
    for v in range(5):
        _eq(o.cells(0, v), z["ghost_U"][v], "ghost U%d" % (v + 1))
    o.recon()
    o.ifbc()
    for d in range(3):
        for side in range(2):
            for v in range(5):
                _eq(o.faces(d, side, v), z["faces_%d" % d][side][v], "faces %d %d %d" % (d, side, v))
    o.dynsmag()
    _eq(o.cells(3), z["mu"], "mu_SGS")
    o.fluxes_only()
    for d in range(3):
        for v in range(5):
            _eq(o.faces(d, 0, v), z["flux_%d" % d][v], "flux %d %d" % (d, v))
    o.evolution(3, 1)
    for v in range(5):
        _eq(o.cells(1, v), z["stage1_Up"][v], "stage-1 Up%d" % (v + 1))
    for stage in (2, 3):
        o.ghost(); o.recon(); o.ifbc(); o.fluxes(); o.evolution(3, stage)
    for v in range(5):
        _eq(o.cells(0, v), z["step_U"][v], "step U%d" % (v + 1))


@pytest.mark.parametrize("name", ["ref_steps_rk3.npz", "ref_steps_rk2chain.npz"])
def test_golden_steps(orc, name):
    z, p = _load(name)
    o = orc.Oracle(p)
    o.set_state(z["state_in"])
    o.step(6)
    _eq(o.state(), z["state_out"], "state after 6 steps")
    assert np.array_equal(o.scalars()[:16], z["scalars"][:16])


def test_golden_filter_minmod_random(orc):
    z, p = _load("ref_misc.npz")
    _eq(orc.Oracle.filter(p, z["field"]), z["filtered"], "filter_")
    lib = orc.Oracle.lib()
    xs = z["xs"]
    mm = np.array([[lib.orc_minmod(x, y) for y in xs] for x in xs])
    _eq(mm, z["minmod"], "minmod")
    seq = [float(z["random_seq"][0])]
    for _ in range(len(z["random_seq"]) - 1):
        seq.append(lib.orc_random(seq[-1]))
    _eq(np.array(seq), z["random_seq"], "Random")
