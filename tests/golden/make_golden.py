"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own serial solver (src/, compiled in place into
oracle/_ref/libfslref.so with the FP64 + zero-fill oracle patch) on small
seeded cases and stores inputs and outputs of every phase:

    python tests/golden/make_golden.py

Needs the reference sources (the oracle Makefile compiles them); the stored
.npz files let the oracle be checked where the reference is absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from tests.helpers import random_state, spatial_params  # noqa: E402


def phases_case(path):
    p = spatial_params(L=10, H=6, D=5, BL_HIG=2)
    s = random_state(p, 101)
    r = orc.RefOracle(p)
    r.set_state(s)
    out = {"state_in": s}
    dist = (1, 4, 11.5, -3.0, 6.25)
    r.set_disturbance(*dist)
    out["disturbance"] = np.array(dist, dtype=np.float64)
    r.ghost()
    out["ghost_U"] = np.stack([r.cells(0, v) for v in range(5)])
    r.recon()
    r.ifbc()
    for d in range(3):
        out["faces_%d" % d] = np.stack([np.stack([r.faces(d, side, v) for v in range(5)]) for side in range(2)])
    r.dynsmag()
    out["mu"] = r.cells(3)
    r.fluxes()
    for d in range(3):
        out["flux_%d" % d] = np.stack([r.faces(d, 0, v) for v in range(5)])
    r.evolution(3, 1)
    out["stage1_Up"] = np.stack([r.cells(1, v) for v in range(5)])
    for stage in (2, 3):
        r.ghost(); r.recon(); r.ifbc(); r.fluxes(); r.evolution(3, stage)
    out["step_U"] = np.stack([r.cells(0, v) for v in range(5)])
    np.savez_compressed(path, params=np.array([repr(p)]), **out)


def steps_case(path, nst):
    p = spatial_params(L=12, H=8, D=6, nStages=nst)
    s = orc.spatial_initial_state(p)
    r = orc.RefOracle(p)
    r.set_state(s)
    r.step(6)
    np.savez_compressed(path, params=np.array([repr(p)]), state_in=s, state_out=r.state(),
                        scalars=r.scalars())


def misc_case(path):
    p = spatial_params(L=7, H=5, D=6)
    r = orc.RefOracle(p)
    rng = np.random.default_rng(7)
    a = rng.standard_normal((p["LEN"] + 2, p["HIG"] + 2, p["DEP"] + 2))
    lib = orc.RefOracle.lib()
    xs = np.concatenate([rng.standard_normal(40), [0.0, -0.0, 1.0, -1.0, 0.25, -0.25, 4.0]])
    mm = np.array([[lib.refh_minmod(x, y) for y in xs] for x in xs])
    seq = [0.317391239817]
    for _ in range(50):
        seq.append(lib.refh_random(seq[-1]))
    np.savez_compressed(path, params=np.array([repr(p)]), field=a, filtered=r.filter(a), xs=xs,
                        minmod=mm, random_seq=np.array(seq))


if __name__ == "__main__":
    orc.build(ref=True)
    phases_case(os.path.join(HERE, "ref_phases.npz"))
    steps_case(os.path.join(HERE, "ref_steps_rk3.npz"), 3)
    steps_case(os.path.join(HERE, "ref_steps_rk2chain.npz"), 2)
    misc_case(os.path.join(HERE, "ref_misc.npz"))
    print("golden vectors written to", HERE)
