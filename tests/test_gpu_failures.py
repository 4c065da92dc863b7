"""Bad states injected on the host come back from the C ABI as
FSL_ERR_NONFINITE, never as a device fault.  Every kernel indexes by the
grid alone, so NaN or a negative density only travels through the
arithmetic: the Courant reduction flags a density that is not positive
(src/helpers.c:23-52 divides by it), and the dt rescale a maximum that is
not positive and finite.  A later good upload clears the flag; with the
time step set again the context steps on as a fresh one."""
import numpy as np
import pytest

from tests.helpers import temporal_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


def _good(fsl, p):
    s, _ = fsl.temporal_state(fsl._as_params(p), 0.4, 1.0, 1e-3, 7)
    return s


def _bad(p, s, var, val):
    b = s.copy().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b[5, 3, var, 4] = val
    return b.ravel()


@pytest.mark.parametrize("var,val", [(0, np.nan), (0, -1.0), (0, 0.0)])
def test_bad_density_fails_the_courant_check(fsl, var, val):
    p = temporal_params(L=16, H=8, D=8)
    d = fsl.Domain(p)
    d.upload_state(_bad(p, _good(fsl, p), var, val))
    with pytest.raises(fsl.FslError) as ex:
        d.check_courant()
    assert ex.value.code == -4
    d.close()


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("var", [0, 4])
def test_nan_state_fails_the_step(fsl, prec, var):
    """NaN in the density or the energy: the fused steps run on, and the
    next sync reports the non-finite state; the context stays usable."""
    p = temporal_params(L=16, H=8, D=8, precision=prec)
    good = _good(fsl, p)
    d = fsl.Domain(p)
    d.upload_state(_bad(p, good, var, np.nan))
    d.step(3)
    with pytest.raises(fsl.FslError) as ex:
        d.sync()
    assert ex.value.code == -4
    # a good state and the time step (which the failed steps made NaN): the
    # context then steps like a fresh one (the temporal setup draws no
    # inflow disturbance, so the skipped draws do not matter)
    d.upload_state(good)
    d.set_time(0, p["deltaT"])
    d.step(2)
    d.sync()
    a = d.download_state()
    d.close()
    ref = fsl.Domain(p)
    ref.upload_state(good)
    ref.step(2)
    b = ref.download_state()
    ref.close()
    assert np.array_equal(a, b)
