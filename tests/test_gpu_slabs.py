"""x-slab decomposition on the GPU: the reach of one step and of one stage,
and slabs that must reproduce the undivided domain bit for bit (FP64, both
reconstructions), with overlap planes exchanged once per step or after every
stage and staged through host or device memory, and two gloo ranks sharing
the GPU (their kernels never wait on one another: the exchange is on the
host)."""
import os
import socket
import sys

import numpy as np
import pytest

from tests.helpers import max_ulp, random_state, spatial_params, temporal_params

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def fsl():
    import freeshearlayer_b200 as fsl
    return fsl


def _same(a, b, what):
    if not np.array_equal(a, b):
        raise AssertionError("%s: max |d| %g, max ulp %d" % (what, np.max(np.abs(a - b)), max_ulp(a, b)))


def _case(fsl, setup, recon=0, L=48, H=12, D=16):
    if setup == 0:
        p = spatial_params(L=L, H=H, D=D, recon=recon)
        s = random_state(p, 31)
    else:
        p = temporal_params(L=L, H=H, D=D, recon=recon)
        s, _ = fsl.temporal_state(fsl._as_params(p), 0.4, 1.0, 2e-2, 7)
    return p, s


def _whole(fsl, p, s, steps):
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step(steps)
    out = d.download_state()
    dt = d.info().deltaT
    d.close()
    return out, dt


@pytest.mark.parametrize("setup", [0, 1])
@pytest.mark.parametrize("recon", [0, 1])
def test_reach_of_one_step(fsl, recon, setup):
    """A change in one plane moves no plane farther than RADIUS in one step
    (the Courant maximum held fixed, so that deltaT is the same)."""
    from freeshearlayer_b200.slabs import RADIUS
    p, s = _case(fsl, setup, recon, L=40)
    P = p["HIG"] * 5 * p["DEP"]
    base = s.reshape(p["LEN"], P)
    pert = base.copy()
    mid = 20
    pert[mid - 1] *= 1.0 + 1e-3 * np.random.default_rng(3).random(P)
    outs = []
    for st in (base, pert):
        d = fsl.Domain(p)
        d.upload_state(st.ravel())
        d.courant_prepare()
        d.set_courant_max(1.0)
        d.step(1)
        outs.append(d.download_state().reshape(p["LEN"], P))
        d.close()
    changed = np.nonzero(np.any(outs[0] != outs[1], axis=1))[0] + 1
    reach = int(np.max(np.abs(changed - mid)))
    print("reach recon=%d setup=%d: %d" % (recon, setup, reach))
    assert reach <= RADIUS[recon], (reach, changed)
    assert reach >= RADIUS[recon] - 2, (reach, changed)   # the bound is not loose


@pytest.mark.parametrize("setup", [1, 0])
@pytest.mark.parametrize("nslabs", [2, 3])
def test_slabs_fused_bit_identical(fsl, setup, nslabs):
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, setup)
    ref, dt = _whole(fsl, p, s, 10)
    with SlabSet(p, nslabs) as ss:
        ss.upload_state(s)
        ss.step(10)
        got = ss.download_state()
        assert all(d.info().deltaT == dt for d in ss.domains)
    _same(got, ref, "%d slabs after 10 steps" % nslabs)


def test_slabs_ppm_bit_identical(fsl):
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, 1, recon=1, L=44)
    ref, _ = _whole(fsl, p, s, 6)
    with SlabSet(p, 2) as ss:
        ss.upload_state(s)
        ss.step(6)
        got = ss.download_state()
    _same(got, ref, "PPM slabs after 6 steps")


def _perturbed_reach(a, b, mid):
    changed = np.nonzero(np.any(a != b, axis=1))[0] + 1
    return int(np.max(np.abs(changed - mid)))


@pytest.mark.parametrize("recon", [0, 1])
def test_reach_of_one_stage(fsl, recon):
    """A change in one plane of U^n moves no plane of the stage-1 output
    farther than STAGE_RADIUS (through the x-stencil and the SGS viscosity),
    and a change in one plane of the stage-1 output moves no plane of the
    stage-2 output farther either."""
    from freeshearlayer_b200.slabs import STAGE_RADIUS
    p, s = _case(fsl, 1, recon, L=40)
    P = p["HIG"] * 5 * p["DEP"]
    L, mid = p["LEN"], 20
    rng = np.random.default_rng(3)
    base = s.reshape(L, P)
    pert = base.copy()
    pert[mid - 1] *= 1.0 + 1e-3 * rng.random(P)
    f1 = 1.0 + 1e-3 * rng.random(P)
    st1, st2 = [], []
    for st in (base, pert, base):
        d = fsl.Domain(p)
        d.upload_state(st.ravel())
        d.courant_prepare()
        d.set_courant_max(1.0)
        d.step_stage()
        st1.append(d.get_planes(1, L, np.empty(L * P)).reshape(L, P))
        if len(st1) == 3:           # perturb the stage state itself
            q = d.get_planes(mid, 1, np.empty(P)) * f1
            d.set_planes(mid, 1, q)
        d.step_stage()
        st2.append(d.get_planes(1, L, np.empty(L * P)).reshape(L, P))
        d.step_stage()
        d.close()
    r1 = _perturbed_reach(st1[0], st1[1], mid)
    r2 = _perturbed_reach(st2[0], st2[2], mid)
    print("stage reach recon=%d: stage 1 %d, stage 2 %d" % (recon, r1, r2))
    assert 2 <= r1 <= STAGE_RADIUS[recon]
    assert 2 <= r2 <= STAGE_RADIUS[recon]


@pytest.mark.parametrize("setup,recon,nslabs", [(1, 0, 2), (1, 0, 3), (0, 0, 3), (1, 1, 3), (0, 1, 2)])
def test_stage_exchange_bit_identical(fsl, setup, recon, nslabs):
    """Overlap planes refreshed after every stage (4 planes instead of 8 or
    10): the owned planes stay bit-identical to the undivided domain."""
    from freeshearlayer_b200.slabs import STAGE_RADIUS, SlabSet
    p, s = _case(fsl, setup, recon, L=44)
    ref, dt = _whole(fsl, p, s, 8)
    with SlabSet(p, nslabs, exchange="stage") as ss:
        assert ss.W == STAGE_RADIUS[recon]
        ss.upload_state(s)
        ss.step(8)
        got = ss.download_state()
        assert all(d.info().deltaT == dt for d in ss.domains)
    _same(got, ref, "%d slabs, per-stage exchange, recon %d" % (nslabs, recon))


def test_stage_exchange_device_staging_fp32(fsl):
    """Per-stage exchange through CUDA tensors, FP32 bulk: agreement to
    rounding (the x-march starts at other planes)."""
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, 1)
    p = dict(p, precision=1)
    ref, _ = _whole(fsl, p, s, 8)
    with SlabSet(p, 3, staging="device", exchange="stage") as ss:
        ss.upload_state(s)
        ss.step(8)
        got = ss.download_state()
    a = got.reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b = ref.reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    for v in (0, 4):
        assert np.linalg.norm(a[:, :, v] - b[:, :, v]) / np.linalg.norm(b[:, :, v]) < 1e-7


def _closure_setup(fsl, d):
    dU = 2.0 * 0.4 * (1.4 * 1e5) ** 0.5
    d.closure_set_scales(1.0 / dU, 1.0)
    d.closure_set_weights(fsl.closure_weights())


@pytest.mark.parametrize("prec,sgs,recon", [(0, 0, 0), (0, 0, 1), (1, 0, 0), (1, 1, 0)])
def test_step_stage_equals_step(fsl, prec, sgs, recon):
    """Three stage calls do exactly what one fsl_step does."""
    p, s = _case(fsl, 1, recon)
    p = dict(p, precision=prec, sgs=sgs)
    outs = []
    for staged in (False, True):
        d = fsl.Domain(p)
        if sgs:
            _closure_setup(fsl, d)
        d.upload_state(s)
        for _ in range(4):
            if staged:
                for _s in range(3):
                    d.step_stage()
            else:
                d.step(1)
        outs.append((d.download_state(), d.info().deltaT))
        d.close()
    _same(outs[1][0], outs[0][0], "stage calls vs fsl_step")
    assert outs[1][1] == outs[0][1]


def test_step_stage_protocol(fsl):
    p, s = _case(fsl, 1, L=32)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step_stage()
    with pytest.raises(fsl.FslError):
        d.step(1)                   # a step is in progress
    with pytest.raises(fsl.FslError):
        d.step_phased(1)
    with pytest.raises(fsl.FslError):
        d.set_courant_max(1.0)      # the final stage accumulates into it
    with pytest.raises(fsl.FslError):
        d.check_courant()
    d.upload_state(s)               # abandons it (its dt rescale and step count stand)
    d.step(1)
    a = d.download_state()
    d.close()
    d = fsl.Domain(p)               # the same begun steps, the first one completed
    d.upload_state(s)
    d.step(1)
    d.upload_state(s)
    d.step(1)
    ref = d.download_state()
    d.close()
    _same(a, ref, "after an abandoned step")
    q = dict(p, nStages=2)
    d = fsl.Domain(q)
    d.upload_state(s)
    with pytest.raises(fsl.FslError):
        d.step_stage()              # the fused stages are RK3
    d.close()


def test_per_phase_calls_refused_mid_step(fsl):
    """While fsl_step_stage is in the middle of a step, the per-phase entry
    points (which would overwrite the stage buffers the step holds) refuse,
    and the step then completes as if they had not been called."""
    p, s = _case(fsl, 1, L=32)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step_stage()
    for call in (d.ghost_bc, d.reconstruct, d.interface_bc, d.dynamic_smagorinsky, d.fluxes,
                 lambda: d.evolution(1)):
        with pytest.raises(fsl.FslError):
            call()
    d.step_stage()
    d.step_stage()
    ref = fsl.Domain(p)
    ref.upload_state(s)
    ref.step(1)
    _same(d.download_state(), ref.download_state(), "a step with refused per-phase calls in between")
    d.close()
    ref.close()


def test_slab_sums_add_up(fsl):
    """Volume integrals and per-row sums over the owned planes, added across
    slabs, equal the undivided domain's to rounding (another summation
    order); an overlap plane counted twice would be off by far more."""
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, 1)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step(3)
    ref_s, ref_r = d.sums(), d.plane_sums()
    d.close()
    with SlabSet(p, 3) as ss:
        ss.upload_state(s)
        ss.step(3)
        got = ss.sums()
        np.testing.assert_allclose(got[[0, 4]], ref_s[[0, 4]], rtol=1e-12)      # mass, energy
        np.testing.assert_allclose(got, ref_s, rtol=0, atol=1e-12 * np.abs(ref_s).max())
        np.testing.assert_allclose(ss.plane_sums(), ref_r, rtol=1e-12, atol=1e-12 * np.abs(ref_r).max())


def test_slabs_against_the_oracle(fsl, oracle_lib):
    """Three slabs against the CPU oracle of the undivided domain."""
    from freeshearlayer_b200.slabs import SlabSet
    p = temporal_params(L=36, H=8, D=8)
    s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    o = oracle_lib.Oracle(p)
    o.set_state(s)
    o.step(5)
    with SlabSet(p, 3) as ss:
        ss.upload_state(s)
        ss.step(5)
        _same(ss.download_state(), o.state(), "3 slabs vs oracle")


def test_slabs_device_staging(fsl):
    """Overlap planes through CUDA tensors (device pointers through the C
    ABI) and the Courant maximum combined in device memory."""
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, 1)
    ref, _ = _whole(fsl, p, s, 8)
    with SlabSet(p, 3, staging="device") as ss:
        ss.upload_state(s)
        ss.step(8)
        got = ss.download_state()
    _same(got, ref, "device-staged slabs")


def test_slabs_fp32_bulk(fsl):
    """FP32 bulk slabs: the x-march starts at other planes than in the
    undivided domain, so agreement is to rounding, not bitwise."""
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, 1)
    p = dict(p, precision=1)
    ref, _ = _whole(fsl, p, s, 8)
    with SlabSet(p, 2) as ss:
        ss.upload_state(s)
        ss.step(8)
        got = ss.download_state()
    a = got.reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b = ref.reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    for v in (0, 4):
        assert np.linalg.norm(a[:, :, v] - b[:, :, v]) / np.linalg.norm(b[:, :, v]) < 1e-7


def test_slabs_fp32_learned_closure(fsl):
    """FP32 bulk + learned closure (judgements off, which slabs require): the
    closure's features reach one plane, so the owned planes agree with the
    undivided domain to FP32 rounding."""
    from freeshearlayer_b200.slabs import SlabSet
    p, s = _case(fsl, 1)
    p = dict(p, precision=1, sgs=1)
    dU = 2.0 * 0.4 * (1.4 * 1e5) ** 0.5

    def setup(d):
        d.closure_set_scales(1.0 / dU, 1.0)
        d.closure_set_weights(fsl.closure_weights())
        d.closure_judge(0, 1.0)

    d = fsl.Domain(p)
    setup(d)
    d.upload_state(s)
    d.step(6)
    ref = d.download_state()
    d.close()
    with SlabSet(p, 2) as ss:
        for x in ss.domains:
            setup(x)
        ss.upload_state(s)
        ss.step(6)
        got = ss.download_state()
    a = got.reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    b = ref.reshape(p["LEN"], p["HIG"], 5, p["DEP"])
    for v in (0, 4):
        assert np.linalg.norm(a[:, :, v] - b[:, :, v]) / np.linalg.norm(b[:, :, v]) < 1e-7


def test_slab_protocol_errors(fsl):
    p, s = _case(fsl, 1, L=32)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.set_courant_range(9, 24)
    with pytest.raises(fsl.FslError):
        d.step(1)                   # no combined Courant maximum yet
    d.courant_prepare()
    with pytest.raises(fsl.FslError):
        d.step(2)                   # one step per call
    with pytest.raises(fsl.FslError):
        d.set_courant_range(0, 5)
    with pytest.raises(fsl.FslError):
        d.get_planes(30, 5, np.empty(5 * d.plane_size()))
    d.step(1)
    d.close()
    q = dict(p, precision=1, sgs=1)
    d = fsl.Domain(q)
    d.upload_state(s)
    d.set_courant_range(9, 24)
    d.courant_prepare()
    with pytest.raises(fsl.FslError):
        d.step(1)                   # closure judgements would differ between slabs
    d.close()


def test_planes_roundtrip(fsl):
    p, s = _case(fsl, 1, L=20)
    d = fsl.Domain(p)
    d.upload_state(s)
    P = d.plane_size()
    got = d.get_planes(5, 3, np.empty(3 * P))
    _same(got, s[4 * P:7 * P], "planes 5..7")
    new = s.copy()
    new[9 * P:12 * P] *= 1.01
    d.set_planes(10, 3, np.ascontiguousarray(new[9 * P:12 * P]))
    _same(d.download_state(), new, "after set_planes")
    d.close()


def test_planes_async_roundtrip(fsl):
    """The stream-ordered plane transfers: CUDA tensors, ordered on the
    domain's stream."""
    import torch
    p, s = _case(fsl, 1, L=20)
    d = fsl.Domain(p)
    d.upload_state(s)
    P = d.plane_size()
    buf = torch.empty(3 * P, dtype=torch.float64, device="cuda")
    d.get_planes_async(5, 3, buf)
    d.sync()
    _same(buf.cpu().numpy(), s[4 * P:7 * P], "planes 5..7, queued")
    buf.mul_(1.01)
    torch.cuda.synchronize()
    d.set_planes_async(10, 3, buf)
    new = s.copy()
    new[9 * P:12 * P] = s[4 * P:7 * P] * 1.01
    _same(d.download_state(), new, "after a queued set")
    d.close()


def _free_port() -> int:
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank_main(rank, world, port, q, exchange="step"):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import freeshearlayer_b200 as fsl
    from freeshearlayer_b200.slabs import DistributedSlab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        p, s = _case(fsl, 1)
        ds = DistributedSlab(p, exchange=exchange)
        ds.upload_state(s)
        ds.step(6)
        full = ds.gather_state(0)
        q.put((rank, None if full is None else full.tobytes()))
        ds.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("exchange", ["step", "stage"])
def test_distributed_slabs_gloo_one_gpu(fsl, exchange):
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q, exchange)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for pr in procs:
        pr.join(60)
        assert pr.exitcode == 0
    full = [r[1] for r in res if r[0] == 0][0]
    p, s = _case(fsl, 1)
    ref, _ = _whole(fsl, p, s, 6)
    _same(np.frombuffer(full, np.float64), ref, "two gloo ranks")


def _nccl_one_rank(port, q, exchange="step"):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import freeshearlayer_b200 as fsl
    from freeshearlayer_b200.slabs import DistributedSlab
    torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    try:
        p, s = _case(fsl, 1)
        ds = DistributedSlab(p, exchange=exchange)
        assert ds.on_device
        ds.upload_state(s)
        ds.step(4)
        full = ds.gather_state(0)
        q.put((full.tobytes(), ds.sums().tobytes()))
        ds.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("exchange", ["step", "stage"])
def test_distributed_slab_nccl_one_rank(fsl, exchange):
    """The NCCL branch of the driver (device buffers, the Courant maximum and
    the integrals all-reduced in device memory) on a one-rank group: the
    undivided domain."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pr = ctx.Process(target=_nccl_one_rank, args=(_free_port(), q, exchange))
    pr.start()
    full, sums = q.get(timeout=300)
    pr.join(60)
    assert pr.exitcode == 0
    p, s = _case(fsl, 1)
    d = fsl.Domain(p)
    d.upload_state(s)
    d.step(4)
    ref, ref_sums = d.download_state(), d.sums()
    d.close()
    _same(np.frombuffer(full, np.float64), ref, "one NCCL rank")
    _same(np.frombuffer(sums, np.float64), ref_sums, "integrals, one NCCL rank")
