"""GPU parity: every phase of the CUDA path against the CPU oracle, through
the C ABI.  The plain method (FP64) must be bit-identical to the oracle, which
itself is bit-identical to the reference's serial code (test_oracle_vs_ref)."""
import numpy as np
import pytest

from tests.helpers import max_ulp, per_var_rel_l2, random_state, spatial_params, temporal_params

pytestmark = pytest.mark.gpu

PARITY_RTOL = 1e-10  # relative L2 per conserved variable after N steps (plain FP64)


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


def _pair(fsl, oracle_lib, p, state):
    o = oracle_lib.Oracle(p)
    o.set_state(state)
    d = fsl.Domain(p)
    d.upload_state(state)
    return o, d


def _assert_same(a, b, what):
    assert a.shape == b.shape, what
    if not np.array_equal(a, b, equal_nan=True):
        raise AssertionError("%s differs: max |d| = %g, max ulp = %d" %
                             (what, np.nanmax(np.abs(a - b)), max_ulp(a, b)))


@pytest.mark.parametrize("setup", [0, 1])
def test_upload_download_roundtrip(fsl, oracle_lib, setup):
    p = spatial_params() if setup == 0 else temporal_params()
    s = random_state(p, 3)
    d = fsl.Domain(p)
    d.upload_state(s)
    _assert_same(d.download_state(), s, "state")


@pytest.mark.parametrize("setup", [0, 1])
def test_phase_ghost(fsl, oracle_lib, setup):
    p = spatial_params() if setup == 0 else temporal_params()
    s = random_state(p, 4)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.ghost(); d.ghost_bc()
    for v in range(5):
        _assert_same(d.cells(0, v), o.cells(0, v), "U%d after ghost fill" % (v + 1))


@pytest.mark.parametrize("setup", [0, 1])
def test_phase_reconstruct_and_interface(fsl, oracle_lib, setup):
    p = spatial_params() if setup == 0 else temporal_params()
    s = random_state(p, 5)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.set_disturbance(1, 4, 12.5, -3.25, 7.0)
    d.set_disturbance(1, 4, 12.5, -3.25, 7.0)
    o.ghost(); d.ghost_bc()
    o.recon(); d.reconstruct()
    o.ifbc(); d.interface_bc()
    for dd in range(3):
        for side in range(2):
            for v in range(5):
                _assert_same(d.faces(dd, side, v), o.faces(dd, side, v),
                             "face dir %d side %d var %d" % (dd, side, v))


def test_phase_interface_wrapped_block(fsl, oracle_lib):
    """Disturbance span with k_max <= k_min wraps around (src/bounCondOnInterfaces.c:134-138)."""
    p = spatial_params(D=8)
    s = random_state(p, 6)
    for kmin, kmax in [(5, 2), (3, 3), (0, 8)]:
        o, d = _pair(fsl, oracle_lib, p, s)
        o.set_disturbance(kmin, kmax, 20.0, 5.0, -5.0)
        d.set_disturbance(kmin, kmax, 20.0, 5.0, -5.0)
        o.ghost(); d.ghost_bc(); o.recon(); d.reconstruct(); o.ifbc(); d.interface_bc()
        for v in range(5):
            _assert_same(d.faces(0, 0, v), o.faces(0, 0, v), "inflow face var %d" % v)


@pytest.mark.parametrize("setup", [0, 1])
def test_phase_dynamic_smagorinsky(fsl, oracle_lib, setup):
    p = spatial_params() if setup == 0 else temporal_params()
    s = random_state(p, 7)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.ghost(); d.ghost_bc()
    o.dynsmag(); d.dynamic_smagorinsky()
    mu_o, mu_d = o.cells(3), d.cells(3)
    assert np.count_nonzero(mu_o) > 0
    _assert_same(mu_d, mu_o, "mu_SGS")


@pytest.mark.parametrize("setup", [0, 1])
def test_phase_fluxes_and_evolution(fsl, oracle_lib, setup):
    p = spatial_params() if setup == 0 else temporal_params()
    s = random_state(p, 8)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.set_disturbance(0, 3, 10.0, 2.0, -1.0)
    d.set_disturbance(0, 3, 10.0, 2.0, -1.0)
    for stage in (1, 2, 3):
        o.ghost(); d.ghost_bc()
        o.recon(); d.reconstruct()
        o.ifbc(); d.interface_bc()
        if stage == 1:
            o.dynsmag(); d.dynamic_smagorinsky()
        o.fluxes_only(); d.fluxes()
        for dd in range(3):
            for v in range(5):
                _assert_same(d.faces(dd, 0, v), o.faces(dd, 0, v), "flux dir %d var %d stage %d" % (dd, v, stage))
        o.evolution(3, stage); d.evolution(stage)
        for v in range(5):
            _assert_same(d.cells(0, v), o.cells(0, v), "U%d after stage %d" % (v + 1, stage))
            _assert_same(d.cells(1, v), o.cells(1, v), "Up%d after stage %d" % (v + 1, stage))


@pytest.mark.parametrize("setup,cfl", [(0, 0), (1, 1)])
def test_check_courant(fsl, oracle_lib, setup, cfl):
    p = spatial_params(cfl_mode=cfl) if setup == 0 else temporal_params()
    s = random_state(p, 9)
    o, d = _pair(fsl, oracle_lib, p, s)
    mo = o.check_courant()
    md, dt = d.check_courant()
    assert md == mo
    assert dt == o.scalars()[0]


@pytest.mark.parametrize("nst", [3, 2])
def test_steps_phased_spatial(fsl, oracle_lib, nst):
    """Whole steps of the reference spatial case (disturbance RNG included);
    nStages = 2 runs the reference's RK2-then-RK3 chain (src/evolution.c:19-23)."""
    p = spatial_params(L=16, H=8, D=8, nStages=nst)
    from oracle.oracle import spatial_initial_state
    s = spatial_initial_state(p)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.step(6); d.step_phased(6)
    _assert_same(d.download_state(), o.state(), "state after 6 steps")
    info = d.info()
    sc = o.scalars()
    assert info.deltaT == sc[0] and info.X == sc[4] and info.step == 6


def test_steps_phased_temporal(fsl, oracle_lib):
    p = temporal_params(L=16, H=8, D=8)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.step(5); d.step_phased(5)
    _assert_same(d.download_state(), o.state(), "state after 5 steps")


@pytest.mark.parametrize("setup", [0, 1])
def test_steps_fused(fsl, oracle_lib, setup):
    """fsl_step (the fused path) against the oracle, several steps."""
    if setup == 0:
        p = spatial_params(L=20, H=10, D=12)
        from oracle.oracle import spatial_initial_state
        s = spatial_initial_state(p)
    else:
        p = temporal_params(L=24, H=12, D=16)
        s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.step(8); d.step(8)
    a, b = d.download_state(), o.state()
    errs = per_var_rel_l2(a, b, p)
    assert max(errs) <= PARITY_RTOL, errs
    _assert_same(a, b, "state after 8 fused steps")


FP32_RTOL = 1e-5  # FP32 bulk: relative L2 of rho and E against the FP64 oracle after 8 steps


@pytest.mark.parametrize("setup", [0, 1])
def test_steps_fp32_bulk(fsl, oracle_lib, setup):
    """FP32 reconstruction/fluxes with FP64 stage accumulation against the
    FP64 oracle.  rho and E within FP32_RTOL; the momenta, normalised by the
    largest momentum magnitude, within 1e-4."""
    if setup == 0:
        p = spatial_params(L=20, H=10, D=12)
        from oracle.oracle import spatial_initial_state
        s = spatial_initial_state(p)
    else:
        p = temporal_params(L=24, H=12, D=16)
        s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    d = fsl.Domain(dict(p, precision=1))
    d.upload_state(s)
    o.step(8)
    d.step(8)
    a = d.download_state().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b = o.state().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    assert np.all(np.isfinite(a))
    errs = per_var_rel_l2(a, b, p)
    assert errs[0] < FP32_RTOL and errs[4] < FP32_RTOL, errs
    mscale = max(np.linalg.norm(b[:, :, v]) for v in (1, 2, 3))
    for v in (1, 2, 3):
        assert np.linalg.norm(a[:, :, v] - b[:, :, v]) / mscale < 1e-4, (v, errs)


def test_sums_and_plane_sums(fsl, oracle_lib):
    p = temporal_params(L=16, H=8, D=8)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    o, d = _pair(fsl, oracle_lib, p, s)
    np.testing.assert_allclose(d.sums(), o.sums(), rtol=1e-13)
    np.testing.assert_allclose(d.plane_sums(), o.plane_sums(), rtol=1e-12)


def _ppm_case(oracle_lib, setup):
    p = (spatial_params(L=12, H=10, D=9) if setup == 0 else temporal_params(L=16, H=10, D=12))
    p = dict(p, recon=1)
    s = random_state(p, 15) if setup == 0 else oracle_lib.Oracle.temporal_state(p, 0.4, amp=0.02)[0]
    return p, s


@pytest.mark.parametrize("setup", [0, 1])
def test_ppm_reconstruct_and_steps(fsl, oracle_lib, setup):
    """PPM (project extension): the per-phase face states, and whole steps of
    the fused stage kernel (fsl_step) and of the per-phase kernels, all
    bit-identical to the oracle's restatement.  Planes per block 1, 3 and 32
    put the x-march's prologue (the reconstruction of the cell before the
    block's first face) at every position, boundary cells included."""
    p, s = _ppm_case(oracle_lib, setup)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.ghost(); d.ghost_bc()
    o.recon(); d.reconstruct()
    for dd in range(3):
        for side in range(2):
            for v in range(5):
                _assert_same(d.faces(dd, side, v), o.faces(dd, side, v), "PPM face dir %d side %d var %d" % (dd, side, v))
    o2 = oracle_lib.Oracle(p)
    o2.set_state(s)
    o2.step(4)
    ref = o2.state()
    for rows, seg in ((16, 1), (16, 3), (16, 32), (8, 3), (12, 5)):
        d2 = fsl.Domain(p)
        d2.tune(d2.TUNE_STAGE_ROWS, rows)
        d2.tune(d2.TUNE_STAGE_SEG, seg)
        d2.upload_state(s)
        d2.step(4)
        _assert_same(d2.download_state(), ref, "state after 4 fused PPM steps, %d rows, %d planes per block"
                     % (rows, seg))
        d2.close()
    d3 = fsl.Domain(p)
    d3.upload_state(s)
    d3.step_phased(4)
    _assert_same(d3.download_state(), ref, "state after 4 per-phase PPM steps")
    d3.close()


@pytest.mark.parametrize("setup,rows", [(0, 16), (1, 16), (1, 8), (1, 12)])
def test_ppm_fp32_bulk(fsl, oracle_lib, setup, rows):
    """PPM with the FP32 bulk (each tile shape) against the FP64 oracle after
    8 steps: rho and E within FP32_RTOL relative L2, the momenta within 1e-4
    of the largest momentum norm (the FP32-bulk bar of the reference scheme)."""
    p, s = _ppm_case(oracle_lib, setup)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(8)
    d = fsl.Domain(dict(p, precision=1))
    d.tune(d.TUNE_STAGE_ROWS, rows)
    d.upload_state(s)
    d.step(8)
    a = d.download_state().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b = o.state().reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    assert np.all(np.isfinite(a))
    errs = per_var_rel_l2(a, b, p)
    assert errs[0] < FP32_RTOL and errs[4] < FP32_RTOL, errs
    mscale = max(np.linalg.norm(b[:, :, v]) for v in (1, 2, 3))
    for v in (1, 2, 3):
        assert np.linalg.norm(a[:, :, v] - b[:, :, v]) / mscale < 1e-4, (v, errs)


def test_c1_config_200_steps(fsl, oracle_lib):
    """The CPU-runnable configuration at full size: temporal shear layer
    64x32x32 on 2pi x pi x pi, Mc 0.4, Re_dw0 500, noise 1e-3 dU, minmod
    characteristic reconstruction, dynamic Smagorinsky, RK3 at acoustic CFL
    0.5, 200 fused steps: all five conserved variables bit-identical to the
    oracle (the stated bar is 1e-10 relative L2)."""
    p = temporal_params(L=64, H=32, D=32, Mc=0.4, Re=500.0)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4, amp=1e-3)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.step(200)
    d.step(200)
    a, b = d.download_state(), o.state()
    errs = per_var_rel_l2(a, b, p)
    assert max(errs) <= PARITY_RTOL, errs
    _assert_same(a, b, "state after 200 steps")


@pytest.mark.parametrize("setup", [0, 1])
@pytest.mark.parametrize("sgs", [2, 3])
def test_steps_static_smagorinsky_and_no_sgs(fsl, oracle_lib, setup, sgs):
    """The static Smagorinsky model (sgs = 2: the reference's
    DynamicSmagorinskySGS 0 branch, rho_face Cs DD |S|_face per face,
    src/fluxes.c:193-205, :362-374, :533-545) and no SGS model (sgs = 3):
    whole fused steps (each tile shape) and per-phase steps bit-identical to
    the oracle, whose static branch is pinned to the reference's own
    (tests/test_oracle_vs_ref.py)."""
    if setup == 0:
        p = spatial_params(L=20, H=10, D=12, sgs=sgs)
        from oracle.oracle import spatial_initial_state
        s = spatial_initial_state(p)
    else:
        p = temporal_params(L=24, H=12, D=16, sgs=sgs, Re=20000.0)
        s, _ = oracle_lib.Oracle.temporal_state(p, 0.4, amp=0.05)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(6)
    ref = o.state()
    for rows in (16, 12, 8):
        d = fsl.Domain(p)
        d.tune(d.TUNE_STAGE_ROWS, rows)
        d.upload_state(s)
        d.step(6)
        _assert_same(d.download_state(), ref, "fused steps, sgs %d, %d rows" % (sgs, rows))
        d.close()
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step_phased(6)
    _assert_same(d.download_state(), ref, "per-phase steps, sgs %d" % sgs)
    d.close()
    # the model matters: the dynamic procedure's steps differ
    q = oracle_lib.Oracle(dict(p, sgs=0))
    q.set_state(s)
    q.step(6)
    assert not np.array_equal(q.state(), ref)


def test_static_smagorinsky_ppm_and_fp32(fsl, oracle_lib):
    """Static Smagorinsky with PPM reconstruction (bit-identical to the
    oracle's restatement) and in the FP32 bulk (rho and E within FP32_RTOL of
    the FP64 oracle after 8 steps)."""
    p = temporal_params(L=16, H=10, D=12, sgs=2, Re=20000.0, recon=1)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4, amp=0.02)
    o, d = _pair(fsl, oracle_lib, p, s)
    o.step(4)
    d.step(4)
    _assert_same(d.download_state(), o.state(), "static Smagorinsky + PPM, 4 steps")
    p32 = dict(p, recon=0)
    o = oracle_lib.Oracle(p32)
    o.set_state(s)
    o.step(8)
    d = fsl.Domain(dict(p32, precision=1))
    d.upload_state(s)
    d.step(8)
    errs = per_var_rel_l2(d.download_state(), o.state(), p32)
    assert errs[0] < FP32_RTOL and errs[4] < FP32_RTOL, errs


# (24, 33, 65) and (28, 20, 65): blocks whose segments are 1 to 3 planes long
# (the halo sweeps run one plane ahead, so the shortest segments matter)
@pytest.mark.parametrize("setup,grid", [(1, (24, 12, 16)), (1, (40, 20, 40)), (1, (33, 17, 33)),
                                        (1, (20, 16, 32)), (0, (20, 10, 12)), (0, (18, 33, 35)),
                                        (1, (24, 33, 65)), (0, (28, 20, 65))])
@pytest.mark.parametrize("sgs", [0, 2])
def test_fp32_full_lane_tile_matches_ring_tile(fsl, oracle_lib, setup, grid, sgs):
    """The FP32 bulk's full-lane persistent stage kernel (rows 0, the default)
    against the ring-tile kernel (rows 16) on grids whose extents are and are
    not multiples of the 16 x 32 tile (partial tiles, a ghost row or column
    as the halo, tiles narrower than the halo work), in both setups, with the
    dynamic and the static SGS model: the same steps to FP32 rounding, and
    both within FP32_RTOL of the FP64 oracle for rho and E."""
    L, H, D = grid
    if setup == 0:
        p = spatial_params(L=L, H=H, D=D, sgs=sgs)
        from oracle.oracle import spatial_initial_state
        s = spatial_initial_state(p)
    else:
        p = temporal_params(L=L, H=H, D=D, sgs=sgs, Re=5000.0)
        s, _ = oracle_lib.Oracle.temporal_state(p, 0.4, amp=0.02)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(6)
    ref = o.state()
    out = {}
    for rows in (0, 16):
        d = fsl.Domain(dict(p, precision=1))
        d.tune(d.TUNE_STAGE_ROWS, rows)
        d.upload_state(s)
        d.step(6)
        out[rows] = d.download_state()
        d.close()
        errs = per_var_rel_l2(out[rows], ref, p)
        assert errs[0] < FP32_RTOL and errs[4] < FP32_RTOL, (rows, errs)
    diff = per_var_rel_l2(out[0], out[16], p)
    assert max(diff[0], diff[1], diff[4]) < 1e-6, diff
    a = out[0].reshape(L, H, 5, D)
    b = out[16].reshape(L, H, 5, D)
    mscale = max(np.linalg.norm(b[:, :, v]) for v in (1, 2, 3))
    for v in (2, 3):
        assert np.linalg.norm(a[:, :, v] - b[:, :, v]) / mscale < 1e-6, (v, diff)


@pytest.mark.parametrize("grid", [(24, 12, 16), (33, 17, 33), (24, 33, 65)])
@pytest.mark.parametrize("sgs", [0, 2])
def test_full_lane_ghost_images_match_ghost_pass(fsl, oracle_lib, grid, sgs):
    """On the temporal setup the full-lane kernel writes its output's ghost
    cells itself, and fsl_step runs the ghost pass only before the first step
    of a call. Six steps in one call (ghost cells from the kernel) must equal
    six calls of one step (ghost cells from the ghost pass before each) bit for
    bit: the kernel's ghost images are exactly the ghost pass's."""
    L, H, D = grid
    p = temporal_params(L=L, H=H, D=D, sgs=sgs, Re=5000.0)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4, amp=0.02)
    out = []
    for calls in ((6,), (1,) * 6):
        d = fsl.Domain(dict(p, precision=1))
        d.tune(d.TUNE_STAGE_ROWS, 0)
        d.upload_state(s)
        for n in calls:
            d.step(n)
        out.append(d.download_state())
        d.close()
    _assert_same(out[0], out[1], "one call of 6 steps vs 6 calls of one step, full-lane tile")


@pytest.mark.parametrize("prec,rows", [(0, None), (1, 16), (1, 0)])
@pytest.mark.parametrize("setup,cfl,Mc", [(0, 0, None), (0, 1, None), (1, 1, 0.4), (1, 1, 0.9)])
def test_fused_courant_maximum_is_the_reduction(fsl, oracle_lib, prec, rows, setup, cfl, Mc):
    """The last stage of a fused step accumulates the Courant maximum of the
    state it writes: it equals the standalone reduction over the same state
    bit for bit, in both setups, both Courant definitions, both precisions
    and both FP32 tiles."""
    if setup == 0:
        p = spatial_params(L=20, H=10, D=12, cfl_mode=cfl)
        from oracle.oracle import spatial_initial_state
        s = spatial_initial_state(p)
    else:
        p = temporal_params(L=40, H=20, D=40, Mc=Mc, Re=5000.0)
        s, _ = oracle_lib.Oracle.temporal_state(p, Mc, amp=0.02)
    d = fsl.Domain(dict(p, precision=prec))
    if rows is not None:
        d.tune(d.TUNE_STAGE_ROWS, rows)
    d.upload_state(s)
    d.step(3)
    fused = d.get_courant_max()
    md, _ = d.check_courant()
    assert fused == md, (fused, md)
    d.close()


@pytest.mark.parametrize("grid", [(128, 20, 40), (256, 33, 65)])
def test_full_lane_long_domains(fsl, oracle_lib, grid):
    """Domains whose full-lane launch splits every tile's planes between a
    head block and the tail blocks (more blocks than tiles), with partial
    tiles: the steps match the ring tile to FP32 rounding and the FP64 oracle
    within the FP32 bar, and repeat bit for bit."""
    L, H, D = grid
    p = temporal_params(L=L, H=H, D=D, Re=5000.0)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4, amp=0.02)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(3)
    ref = o.state()
    out = []
    for rows in (0, 0, 16):
        d = fsl.Domain(dict(p, precision=1))
        d.tune(d.TUNE_STAGE_ROWS, rows)
        d.upload_state(s)
        d.step(3)
        out.append(d.download_state())
        d.close()
        errs = per_var_rel_l2(out[-1], ref, p)
        assert errs[0] < FP32_RTOL and errs[4] < FP32_RTOL, (rows, errs)
    assert np.array_equal(out[0], out[1])
    diff = per_var_rel_l2(out[0], out[2], p)
    assert max(diff[0], diff[1], diff[4]) < 1e-6, diff
