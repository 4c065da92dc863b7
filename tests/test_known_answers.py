"""Known answers that follow from the reference's code itself, on the CPU
oracle: the limiter's closed form (src/reconstruction.c:17-24), the test
filter of a constant field (src/turbulence.c:17-100: the constant to one
rounding of the three 1/3-weighted sums, two cells or more from the zero
bands), and, in the temporal setup (periodic x and z, copied y ghosts), a
uniform flow that every phase leaves uniform (zero flux divergence; the RK
combination only rounds) with no SGS viscosity (M = 0, Cd = -0.5 * 0 /
(0 + 1e-30) clipped to 0, src/turbulence.c:433-442).  The spatial setup's
inflow plane holds its own profile, so a uniform state is not steady
there."""
import numpy as np

from tests.helpers import temporal_params


def _uniform(p, r=1.2, u=150.0, v=-3.0, w=7.0, P=1e5):
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    s = np.empty((L, H, 5, D))
    s[:, :, 0, :] = r
    s[:, :, 1, :] = r * u
    s[:, :, 2, :] = r * v
    s[:, :, 3, :] = r * w
    s[:, :, 4, :] = P / 0.4 + 0.5 * r * (u * u + v * v + w * w)
    return s.ravel()


def test_minmod_closed_form(oracle_lib):
    lib = oracle_lib.Oracle.lib()
    vals = [0.0, -0.0, 1e-300, 0.1, -0.1, 0.25, -0.25, 1.0, -1.0, 3.9, -4.1, 1e3, -1e3]
    for x in vals:
        for y in vals:
            want = 0.0 if x * y <= 0 else np.copysign(min(abs(x), 4.0 * abs(y)), x)
            assert lib.orc_minmod(x, y) == want, (x, y)


def test_filter_of_a_constant_is_the_constant(oracle_lib):
    p = temporal_params(L=16, H=12, D=10)
    a = np.full(oracle_lib.padded_shape(p), 3.5)
    f = oracle_lib.Oracle.filter(p, a)
    assert np.max(np.abs(f[2:-2, 2:-2, 2:-2] - 3.5)) <= np.spacing(3.5)
    assert np.min(f[1, 1:-1, 1:-1]) < 3.0       # the zero band one cell in reaches it


def test_uniform_flow_stays_uniform(oracle_lib):
    p = temporal_params(L=16, H=12, D=10)
    s = _uniform(p)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(3)
    a = o.state().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b = s.reshape(a.shape)
    for q in range(5):
        assert np.max(np.abs(a[:, :, q] - b[:, :, q])) <= 4e-16 * abs(b[0, 0, q, 0]), q


def test_uniform_velocity_has_no_sgs_viscosity(oracle_lib):
    p = temporal_params(L=16, H=12, D=10)
    o = oracle_lib.Oracle(p)
    o.set_state(_uniform(p))
    o.ghost()
    o.dynsmag()
    mu = o.cells(3)
    assert np.all(mu == 0.0), np.max(np.abs(mu))
