"""Pin the oracle: the project's C restatement (oracle/fsl_oracle.c) against the
reference's own serial solver compiled in place (oracle/_ref/libfslref.so),
phase by phase and over whole steps.  FP64 on both sides, no FMA: results
must be bit-identical."""
import numpy as np
import pytest

from tests.helpers import max_ulp, random_state, spatial_params


@pytest.fixture(scope="module")
def orc(oracle_lib):
    if not oracle_lib.ref_available():
        pytest.skip("reference oracle library not built (reference sources absent)")
    return oracle_lib


def _eq(a, b, what):
    if not np.array_equal(a, b, equal_nan=True):
        raise AssertionError("%s: max |d| %g, max ulp %d" % (what, np.nanmax(np.abs(a - b)), max_ulp(a, b)))


def _pair(orc, p, s):
    r = orc.RefOracle(p)
    r.set_state(s)
    o = orc.Oracle(p)
    o.set_state(s)
    return r, o


def test_minmod_and_random(orc):
    r = orc.RefOracle.lib()
    o = orc.Oracle.lib()
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.standard_normal(200), [0.0, -0.0, 1.0, -1.0, 0.25, -0.25, 4.0]])
    for x in xs:
        for y in xs[::7]:
            assert r.refh_minmod(x, y) == o.orc_minmod(x, y)
    x = 0.317391239817
    for _ in range(100):
        a, b = r.refh_random(x), o.orc_random(x)
        assert a == b
        x = a


def test_filter(orc):
    p = spatial_params(L=7, H=5, D=6)
    r = orc.RefOracle(p)
    a = np.random.default_rng(3).standard_normal((p["LEN"] + 2, p["HIG"] + 2, p["DEP"] + 2))
    _eq(orc.Oracle.filter(p, a), r.filter(a), "filter_")


def test_ghost_recon_interface(orc):
    p = spatial_params(L=9, H=8, D=7, BL_HIG=3)
    s = random_state(p, 21)
    r, o = _pair(orc, p, s)
    for kmin, kmax in [(1, 5), (5, 1), (2, 2)]:
        r.set_disturbance(kmin, kmax, 11.0, -4.0, 3.0)
        o.set_disturbance(kmin, kmax, 11.0, -4.0, 3.0)
        r.ghost(); o.ghost()
        for v in range(5):
            _eq(o.cells(0, v), r.cells(0, v), "ghost U%d" % (v + 1))
        r.recon(); o.recon()
        r.ifbc(); o.ifbc()
        for d in range(3):
            for side in range(2):
                for v in range(5):
                    _eq(o.faces(d, side, v), r.faces(d, side, v), "faces %d %d %d" % (d, side, v))


def test_dynamic_smagorinsky(orc):
    p = spatial_params(L=8, H=6, D=7)
    s = random_state(p, 22)
    r, o = _pair(orc, p, s)
    r.ghost(); o.ghost()
    r.dynsmag(); o.dynsmag()
    mu = o.cells(3)
    assert np.count_nonzero(mu) > 0
    _eq(mu, r.cells(3), "mu_SGS")


def test_stages(orc):
    p = spatial_params(L=8, H=6, D=5)
    s = random_state(p, 23)
    r, o = _pair(orc, p, s)
    r.set_disturbance(0, 3, 5.0, 1.0, -2.0)
    o.set_disturbance(0, 3, 5.0, 1.0, -2.0)
    for stage in (1, 2, 3):
        r.ghost(); o.ghost()
        r.recon(); o.recon()
        r.ifbc(); o.ifbc()
        r.fluxes(); o.fluxes()
        for d in range(3):
            for v in range(5):
                _eq(o.faces(d, 0, v), r.faces(d, 0, v), "flux %d %d stage %d" % (d, v, stage))
        r.evolution(3, stage); o.evolution(3, stage)
        for v in range(5):
            _eq(o.cells(0, v), r.cells(0, v), "U%d stage %d" % (v + 1, stage))
            _eq(o.cells(1, v), r.cells(1, v), "Up%d stage %d" % (v + 1, stage))


@pytest.mark.parametrize("nst", [3, 2])
def test_whole_steps(orc, nst):
    """Driver loop incl. Courant rescale and disturbance RNG.  The oracle
    evaluates the SGS viscosity once per step; the reference in every stage."""
    p = spatial_params(L=16, H=8, D=8, nStages=nst)
    s = orc.spatial_initial_state(p)
    r, o = _pair(orc, p, s)
    r.step(12); o.step(12)
    _eq(o.state(), r.state(), "state after 12 steps")
    rs, os_ = r.scalars(), o.scalars()
    assert np.array_equal(rs[:16], os_[:16])


def test_sgs_once_per_step_equals_every_stage(orc):
    p = spatial_params(L=12, H=8, D=6)
    s = random_state(p, 24)
    a = orc.Oracle(p); a.set_state(s)
    b = orc.Oracle(p); b.set_state(s)
    a.step(4); b.step_ref_sgs(4)
    _eq(a.state(), b.state(), "once-per-step SGS")


def test_output_frame(orc, tmp_path):
    """Output() (src/output.c): the restatement's 12 values per cell, written
    by the library's Tecplot writer, give the reference's <step>.plt byte for
    byte (after steps, with the ghost layer the last stage left)."""
    import freeshearlayer_b200 as fsl
    p = spatial_params(L=10, H=8, D=6)
    s = orc.spatial_initial_state(p)
    r, o = _pair(orc, p, s)
    r.step(3); o.step(3)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    assert r.output(str(ref_dir)) == 0
    ref_file = ref_dir / "3.plt"
    mine = tmp_path / "mine.plt"
    fsl.tecplot_write(str(mine), o.output_fields())
    assert mine.read_bytes() == ref_file.read_bytes()


def test_static_smagorinsky_fluxes(orc):
    """The static Smagorinsky branch of the reference's Fluxes()
    (src/fluxes.c:193-205, :362-374, :533-545; dead in src, which hardcodes
    the dynamic procedure, live in src-par/def.h:47) compiled in place with
    the macro set to 0, against the restatement's sgs = 2: every face flux
    bit-identical, and not equal to the dynamic procedure's."""
    p = spatial_params(L=8, H=6, D=5, sgs=2)
    s = random_state(p, 25)
    r, o = _pair(orc, p, s)
    r.set_disturbance(0, 3, 5.0, 1.0, -2.0)
    o.set_disturbance(0, 3, 5.0, 1.0, -2.0)
    for stage in (1, 2, 3):
        r.ghost(); o.ghost()
        r.recon(); o.recon()
        r.ifbc(); o.ifbc()
        r.fluxes_static(); o.fluxes()
        for d in range(3):
            for v in range(5):
                _eq(o.faces(d, 0, v), r.faces(d, 0, v), "static flux %d %d stage %d" % (d, v, stage))
        r.evolution(3, stage); o.evolution(3, stage)
        for v in range(5):
            _eq(o.cells(0, v), r.cells(0, v), "U%d stage %d" % (v + 1, stage))
    # the dynamic procedure gives other fluxes on the same state
    q = orc.Oracle(dict(p, sgs=0))
    q.set_state(s)
    q.set_disturbance(0, 3, 5.0, 1.0, -2.0)
    q.ghost(); q.recon(); q.ifbc(); q.fluxes()
    o2 = orc.Oracle(p)
    o2.set_state(s)
    o2.set_disturbance(0, 3, 5.0, 1.0, -2.0)
    o2.ghost(); o2.recon(); o2.ifbc(); o2.fluxes()
    assert not np.array_equal(q.faces(0, 0, 1), o2.faces(0, 0, 1))


def test_static_smagorinsky_whole_steps(orc):
    """Whole driver steps with the static branch (Courant rescale, disturbance
    draw, three stages): the restatement equals the reference bit for bit."""
    p = spatial_params(L=16, H=8, D=8, sgs=2)
    s = orc.spatial_initial_state(p)
    r, o = _pair(orc, p, s)
    r.step(8); o.step(8)
    _eq(o.state(), r.state(), "static SGS state after 8 steps")


def test_no_sgs_is_static_with_zero_constant(orc):
    """sgs = 3 (no SGS viscosity) equals the static model with Cs = 0."""
    p = spatial_params(L=12, H=8, D=6)
    s = random_state(p, 26)
    a = orc.Oracle(dict(p, sgs=3)); a.set_state(s)
    b = orc.Oracle(dict(p, sgs=2, Cs=0.0)); b.set_state(s)
    a.step(3); b.step(3)
    _eq(a.state(), b.state(), "no SGS vs Cs = 0")
