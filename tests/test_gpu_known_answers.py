"""Known answers through the C ABI on the GPU, in the temporal setup
(periodic x and z, copied y ghosts): a uniform flow stays uniform under
every step path (zero flux divergence; the FP64 RK combination rounds, and
in the FP32 bulk the x-march may contract a block's first face into FMAs
differently from the others, a difference of FP32 rounding), and a uniform
velocity field has no SGS viscosity (src/turbulence.c:433-442)."""
import numpy as np
import pytest

from tests.helpers import temporal_params
from tests.test_known_answers import _uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


# (precision, sgs, recon, relative tolerance per conserved variable after 3 steps)
CASES = [(0, 0, 0, 4e-16), (0, 0, 1, 4e-16), (1, 0, 0, 1e-6), (1, 0, 1, 1e-6), (1, 1, 0, 1e-6)]


@pytest.mark.parametrize("prec,sgs,recon,tol", CASES)
def test_uniform_flow_stays_uniform(fsl, prec, sgs, recon, tol):
    p = temporal_params(L=32, H=20, D=40, precision=prec, sgs=sgs, recon=recon)
    s = _uniform(p)
    d = fsl.Domain(p)
    if sgs:
        d.closure_set_scales(1.0 / (2.0 * 0.4 * (1.4 * 1e5) ** 0.5), 1.0)
        d.closure_set_weights(fsl.closure_weights())
    d.upload_state(s)
    d.step(3)
    a = d.download_state().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    d.close()
    b = s.reshape(a.shape)
    for q in range(5):
        err = np.max(np.abs(a[:, :, q] - b[:, :, q])) / abs(b[0, 0, q, 0])
        assert err <= tol, (q, err)


def test_uniform_velocity_has_no_sgs_viscosity(fsl):
    p = temporal_params(L=16, H=12, D=10)
    d = fsl.Domain(p)
    d.upload_state(_uniform(p))
    d.ghost_bc()
    d.dynamic_smagorinsky()
    mu = d.cells(3)
    d.close()
    assert np.all(mu == 0.0), np.max(np.abs(mu))
