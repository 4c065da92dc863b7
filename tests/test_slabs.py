"""x-slab decomposition, host logic on CPU: the layout, the exchange plan and
the per-step and per-stage protocols (Courant maximum combined across slabs,
overlap planes refreshed from the neighbours) of SlabSet and of
DistributedSlab over gloo ranks, driven on a stand-in context whose stages are
x-stencils of the same reach.  Every owned plane must come out bit-identical
to the undivided domain's."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# sub-steps of the three-point stencil per stage: one stage reaches at most
# STAGE_RADIUS planes, one step RADIUS
TOY_STAGES = {0: (4, 2, 2), 1: (4, 3, 3)}


class ToyDomain:
    """Stand-in for a slab context with the methods the slab drivers use.
    One step: deltaT rescaled to maxCoNum by the Courant maximum (max |u| dt,
    over the Courant range), then three stages, each a few sub-steps of a
    three-point x stencil with the setup's x boundary (periodic in the
    temporal setup; an inflow plane of ones and a zero-gradient outflow in the
    spatial one) and, like the SGS filter's zero bands, a treatment of its own
    for the first and last plane, periodic or not; stages 2 and 3 are combined
    with U^n plane by plane like the RK stages.  After the step the maximum of
    the new state is kept, as the fused final stage does.  get_planes /
    set_planes act on the stage state in the middle of a step."""

    def __init__(self, p):
        from freeshearlayer_b200.slabs import RADIUS, STAGE_RADIUS
        self.L, self.plane = p.LEN, p.HIG * 5 * p.DEP
        self.periodic = p.setup == 1
        self.stages = TOY_STAGES[p.recon]
        assert sum(self.stages) == RADIUS[p.recon] and max(self.stages) == STAGE_RADIUS[p.recon]
        self.u = np.zeros((self.L, self.plane))
        self.v, self.next = None, 0
        self.dt, self.maxco = p.deltaT, p.maxCoNum
        self.co0, self.co1, self.co = 1, self.L, None

    def close(self):
        pass

    def sync(self):
        pass

    def set_courant_range(self, i0, i1):
        self.co0, self.co1, self.co = i0, i1, None

    def upload_state(self, s):
        self.u = np.asarray(s, np.float64).reshape(self.L, self.plane).copy()
        self.co, self.next = None, 0

    def _cur(self):
        return self.v if self.next else self.u

    def get_planes(self, i0, n, out):
        out[:n * self.plane] = self._cur()[i0 - 1:i0 - 1 + n].ravel()
        return out

    def set_planes(self, i0, n, buf):
        self._cur()[i0 - 1:i0 - 1 + n] = np.asarray(buf[:n * self.plane]).reshape(n, self.plane)
        if not self.next and i0 <= self.co1 and i0 + n - 1 >= self.co0:
            self.co = None

    def sums(self):
        return self.u[self.co0 - 1:self.co1].sum(axis=0)[:5]

    def plane_sums(self):
        return self.u[self.co0 - 1:self.co1].sum(axis=0).reshape(-1, 2)

    def _owned_max(self):
        return float(np.max(np.abs(self.u[self.co0 - 1:self.co1]) * self.dt))

    def courant_prepare(self):
        if self.co is None:
            self.co = self._owned_max()

    def get_courant_max(self):
        assert self.co is not None
        return self.co

    def set_courant_max(self, m):
        self.co = m

    def step_stage(self):
        slab = (self.co0, self.co1) != (1, self.L)
        if self.next == 0:
            if slab and self.co is None:
                raise RuntimeError("x-slab: no combined maximum")
            m = self.co if self.co is not None else self._owned_max()
            self.dt = self.dt * (self.maxco / m)
            self.v = self.u.copy()
        s = self.next
        v, c = self.v, self.dt
        for _ in range(self.stages[s]):
            g = np.empty((self.L + 2, self.plane))
            g[1:-1] = v
            if self.periodic:
                g[0], g[-1] = v[-1], v[0]
            else:
                g[0], g[-1] = 1.0, v[-1]
            v = v + c * (g[:-2] - 2.0 * v + g[2:])
            v[0] *= 0.999
            v[-1] *= 1.001
        if s == 1:
            v = 0.75 * self.u + 0.25 * v
        elif s == 2:
            v = self.u / 3.0 + 2.0 / 3.0 * v
        if s == 2:
            self.u, self.v, self.next = v, None, 0
            self.co = self._owned_max()
        else:
            self.v, self.next = v, s + 1

    def step(self, n=1):
        slab = (self.co0, self.co1) != (1, self.L)
        if self.next:
            raise RuntimeError("a step is in progress")
        if slab and (n > 1 or self.co is None):
            raise RuntimeError("x-slab: one step per call, after a combined maximum")
        for _ in range(n):
            for _s in range(3):
                self.step_stage()

    step_phased = step


def _params(setup, L=37, recon=0):
    import freeshearlayer_b200 as fsl
    return fsl.default_params(LEN=L, HIG=3, DEP=2, setup=setup, recon=recon, deltaT=1.0, maxCoNum=0.3)


def _state(p, seed=5):
    rng = np.random.default_rng(seed)
    return 1.0 + 0.5 * rng.random(p.LEN * p.HIG * 5 * p.DEP)


def _whole(p, state, steps):
    d = ToyDomain(p)
    d.upload_state(state)
    for _ in range(steps):
        d.courant_prepare()
        d.set_courant_max(d.get_courant_max())
        d.step(1)
    return d.u.ravel(), d.dt


def test_layout_covers_every_plane_once():
    from freeshearlayer_b200.slabs import exchange_plan, layout
    for periodic in (True, False):
        for L, S, W in [(40, 1, 8), (40, 2, 8), (41, 3, 8), (80, 4, 10), (64, 8, 8)]:
            slabs = layout(L, S, W, periodic)
            owned = np.concatenate([np.arange(s.a, s.b + 1) for s in slabs])
            assert np.array_equal(owned, np.arange(1, L + 1))
            for s in slabs:
                gp = s.global_planes()
                assert len(gp) == s.local_len == len(set(gp.tolist()))
                assert np.array_equal(gp[s.own0 - 1:s.own1], np.arange(s.a, s.b + 1))
                if 1 in gp and L in gp:   # the seam on the local periodic boundary
                    assert gp[0] == 1 and gp[-1] == L
            # every overlap plane is filled from the slab that owns it
            for src, i0, dst, j0, n in exchange_plan(slabs):
                gs = slabs[src].global_planes()[i0 - 1:i0 - 1 + n]
                gd = slabs[dst].global_planes()[j0 - 1:j0 - 1 + n]
                assert np.array_equal(gs, gd)
                assert slabs[src].a <= gs.min() and gs.max() <= slabs[src].b
            if not periodic and S > 1:
                assert slabs[0].wl == 0 and slabs[-1].wr == 0
    with pytest.raises(ValueError):
        layout(20, 4, 8, True)        # slabs thinner than the overlap
    with pytest.raises(ValueError):
        layout(20, 2, 8, True)        # a slab and its overlap cover the domain twice


def test_overlap_below_the_reach_is_refused():
    from freeshearlayer_b200.slabs import SlabSet
    with pytest.raises(ValueError):
        SlabSet(_params(1), 2, overlap=7, domain_factory=ToyDomain)
    with pytest.raises(ValueError):
        SlabSet(_params(1, recon=1, L=60), 2, overlap=9, domain_factory=ToyDomain)


@pytest.mark.parametrize("setup", [1, 0])
@pytest.mark.parametrize("nslabs", [1, 2, 3, 4])
def test_slabset_matches_whole_domain(setup, nslabs):
    from freeshearlayer_b200.slabs import SlabSet
    p = _params(setup)
    s0 = _state(p)
    ref, dt = _whole(p, s0, 6)
    with SlabSet(p, nslabs, domain_factory=ToyDomain) as ss:
        ss.upload_state(s0)
        ss.step(6)
        got = ss.download_state()
        assert all(d.dt == dt for d in ss.domains)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("recon", [0, 1])
@pytest.mark.parametrize("setup", [1, 0])
@pytest.mark.parametrize("nslabs", [2, 3, 4])
def test_stage_exchange_matches_whole_domain(setup, nslabs, recon):
    from freeshearlayer_b200.slabs import STAGE_RADIUS, SlabSet
    p = _params(setup, recon=recon)
    s0 = _state(p)
    ref, dt = _whole(p, s0, 6)
    with SlabSet(p, nslabs, domain_factory=ToyDomain, exchange="stage") as ss:
        assert ss.W == STAGE_RADIUS[recon]
        ss.upload_state(s0)
        ss.step(6)
        got = ss.download_state()
        assert all(d.dt == dt for d in ss.domains)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("setup", [1, 0])
def test_slab_sums_add_up(setup):
    from freeshearlayer_b200.slabs import SlabSet
    p = _params(setup)
    s0 = _state(p)
    whole = ToyDomain(p)
    whole.upload_state(s0)
    with SlabSet(p, 3, domain_factory=ToyDomain) as ss:
        ss.upload_state(s0)
        np.testing.assert_allclose(ss.sums(), whole.sums(), rtol=1e-13)
        np.testing.assert_allclose(ss.plane_sums(), whole.plane_sums(), rtol=1e-13)


def test_stage_overlap_exchanged_once_per_step_goes_wrong():
    """The check has teeth: the narrow per-stage overlap, refreshed only after
    the whole step, is too narrow."""
    from freeshearlayer_b200.slabs import SlabSet
    p = _params(1)
    s0 = _state(p)
    ref, _ = _whole(p, s0, 3)
    with SlabSet(p, 3, domain_factory=ToyDomain, exchange="stage") as ss:
        ss.upload_state(s0)
        for _ in range(3):
            ss.combine_courant()
            for d in ss.domains:
                d.step(1)
            ss.exchange()
        assert not np.array_equal(ss.download_state(), ref)


def test_stage_exchange_arguments():
    from freeshearlayer_b200.slabs import SlabSet
    with pytest.raises(ValueError):
        SlabSet(_params(1), 2, overlap=3, domain_factory=ToyDomain, exchange="stage")
    with pytest.raises(ValueError):
        SlabSet(_params(1), 2, domain_factory=ToyDomain, exchange="plane")
    q = _params(1)
    q.nStages = 2
    with pytest.raises(ValueError):
        SlabSet(q, 2, domain_factory=ToyDomain, exchange="stage")
    with SlabSet(_params(1), 2, domain_factory=ToyDomain, exchange="stage") as ss:
        ss.upload_state(_state(_params(1)))
        with pytest.raises(ValueError):
            ss.step(1, phased=True)


def test_without_exchange_the_slabs_go_wrong():
    """The check has teeth: a slab set that skips the overlap refresh differs."""
    from freeshearlayer_b200.slabs import SlabSet
    p = _params(1)
    s0 = _state(p)
    ref, _ = _whole(p, s0, 4)
    with SlabSet(p, 3, domain_factory=ToyDomain) as ss:
        ss.upload_state(s0)
        for _ in range(4):
            ss.combine_courant()
            for d in ss.domains:
                d.step(1)
        assert not np.array_equal(ss.download_state(), ref)


def test_seam_inside_a_slab_goes_wrong(monkeypatch):
    """The check has teeth: local planes in cyclic order (the periodic seam
    inside the slab, not on its boundary) miss the seam's own treatment."""
    from freeshearlayer_b200 import slabs as S
    p = _params(1)
    s0 = _state(p)
    ref, _ = _whole(p, s0, 3)
    monkeypatch.setattr(S.Slab, "global_planes",
                        lambda self: (np.arange(self.a - self.wl, self.b + self.wr + 1) - 1) % self.LEN + 1)
    with S.SlabSet(p, 3, domain_factory=ToyDomain) as ss:
        ss.upload_state(s0)
        ss.step(3)
        assert not np.array_equal(ss.download_state(), ref)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, setup, steps, q, exchange="step"):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_slabs import ToyDomain, _params, _state
    from freeshearlayer_b200.slabs import DistributedSlab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = _params(setup)
        ds = DistributedSlab(p, domain_factory=ToyDomain, exchange=exchange)
        ds.upload_state(_state(p))
        ds.step(steps)
        full = ds.gather_state(0)
        sums = ds.sums()
        q.put((rank, ds.dom.dt, None if full is None else full.tolist(), sums.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,setup,exchange", [(2, 1, "step"), (3, 1, "step"), (2, 0, "step"), (3, 0, "step"),
                                                  (3, 1, "stage"), (2, 0, "stage")])
def test_distributed_gloo_matches_whole_domain(world, setup, exchange):
    steps = 5
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, setup, steps, q, exchange))
             for r in range(world)]
    for pr in procs:
        pr.start()
    # read before joining: a rank cannot exit while its result is unread in the pipe
    res = sorted((q.get(timeout=120) for _ in range(world)), key=lambda x: x[0])
    for pr in procs:
        pr.join(60)
        assert pr.exitcode == 0
    p = _params(setup)
    ref, dt = _whole(p, _state(p), steps)
    assert all(r[1] == dt for r in res)
    assert np.array_equal(np.array(res[0][2]), ref)
    whole = ToyDomain(p)
    whole.upload_state(ref)
    for r in res:                   # the SUM all-reduce gives every rank the whole
        np.testing.assert_allclose(r[3], whole.sums(), rtol=1e-13)
