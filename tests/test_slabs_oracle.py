"""x-slabs of the real scheme on the CPU: the slab drivers run over contexts
that step with the CPU oracle (the reference's own arithmetic, phase by phase
as src/layer2.c:141-178 orders it), and the owned planes must come out
bit-identical to the oracle's undivided step, deltaT included, with the
overlap exchanged once per step or after every stage, in both setups and
with both reconstructions.  The Courant maximum over a slab's owned planes
is formed here in the oracle's expression order (src/helpers.c:23-52 and the
acoustic variant), so the combined maximum equals the undivided one."""
import numpy as np
import pytest


class OracleDomain:
    """A slab context with the methods the slab drivers use, stepping with
    the oracle: per step the dt rescale from the (combined) Courant maximum,
    the disturbance draw, then three stages of ghost cells, reconstruction,
    interface conditions, SGS viscosity (stage 1), fluxes and evolution."""

    def __init__(self, p):
        from oracle.oracle import Oracle, OrcParams
        self.p = {k: getattr(p, k) for k, _ in OrcParams._fields_}
        self.o = Oracle(self.p)
        self.L, self.H, self.D = self.p["LEN"], self.p["HIG"], self.p["DEP"]
        self.dt = self.p["deltaT"]
        self.co0, self.co1, self.co = 1, self.L, None
        self.next = 0

    def close(self):
        pass

    def sync(self):
        pass

    def set_courant_range(self, i0, i1):
        self.co0, self.co1, self.co = i0, i1, None

    def upload_state(self, s):
        self.o.set_state(np.asarray(s, np.float64))
        self.co, self.next = None, 0

    def _which(self):
        return 1 if self.next else 0    # mid-step: the stage buffer

    def get_planes(self, i0, n, out):
        w = self._which()
        a = np.stack([self.o.cells(w, q)[i0:i0 + n, 1:-1, 1:-1] for q in range(5)], axis=2)
        out[:a.size] = a.ravel()
        return out

    def set_planes(self, i0, n, buf):
        w = self._which()
        a = np.asarray(buf[:n * self.H * 5 * self.D]).reshape(n, self.H, 5, self.D)
        for q in range(5):
            c = self.o.cells(w, q)
            c[i0:i0 + n, 1:-1, 1:-1] = a[:, :, q, :]
            self.o.set_cells(w, q, c)
        if not self.next and i0 <= self.co1 and i0 + n - 1 >= self.co0:
            self.co = None

    def _owned_max(self):
        U = [self.o.cells(0, q)[self.co0:self.co1 + 1, 1:-1, 1:-1] for q in range(5)]
        dtx, dty, dtz = self.dt / self.p["deltaX"], self.dt / self.p["deltaY"], self.dt / self.p["deltaZ"]
        R = U[0]
        if self.p["cfl_mode"] == 1:
            ir = 1.0 / R
            u, v, w = U[1] * ir, U[2] * ir, U[3] * ir
            P = (U[4] - 0.5 * R * (u * u + v * v + w * w)) * 0.4
            Cs = np.sqrt(1.4 * P * ir)
            co = (np.abs(u) + Cs) * dtx + (np.abs(v) + Cs) * dty + (np.abs(w) + Cs) * dtz
        else:
            co = U[1] / R * dtx
        return max(0.0, float(np.max(co)))

    def courant_prepare(self):
        if self.co is None:
            self.co = self._owned_max()

    def get_courant_max(self):
        return self.co

    def set_courant_max(self, m):
        self.co = m

    def step_stage(self):
        o = self.o
        if self.next == 0:
            if self.co is None:
                raise RuntimeError("no combined Courant maximum")
            self.dt = self.dt * (self.p["maxCoNum"] / self.co)
            o.set_dt(self.dt)
            o.disturb()
            self.next = 1
        s = self.next
        o.ghost()
        o.recon()
        o.ifbc()
        if s == 1:
            o.dynsmag()
        o.fluxes_only()
        o.evolution(3, s)
        self.next = 0 if s == 3 else s + 1
        if s == 3:
            self.co = None

    def step(self, n=1):
        for _ in range(n):
            self.courant_prepare()
            for _s in range(3):
                self.step_stage()

    step_phased = step


def _case(oracle_lib, setup, recon, L=36):
    from tests.helpers import spatial_params, temporal_params
    if setup == 1:
        p = temporal_params(L=L, H=8, D=8, recon=recon)
        s, _ = oracle_lib.Oracle.temporal_state(p, 0.4)
    else:
        from oracle.oracle import spatial_initial_state
        p = spatial_params(L=L, H=8, D=6, recon=recon)
        s = spatial_initial_state(p)
    return p, s


@pytest.mark.parametrize("exchange", ["step", "stage"])
@pytest.mark.parametrize("recon", [0, 1])
@pytest.mark.parametrize("setup", [1, 0])
def test_oracle_slabs_bit_identical(oracle_lib, setup, recon, exchange):
    import freeshearlayer_b200 as fsl
    from freeshearlayer_b200.slabs import SlabSet
    L = 44 if (recon == 1 and exchange == "step") else 36
    p, s = _case(oracle_lib, setup, recon, L)
    ref = oracle_lib.Oracle(p)
    ref.set_state(s)
    ref.step(4)
    with SlabSet(fsl._as_params(p), 3, domain_factory=OracleDomain, exchange=exchange) as ss:
        ss.upload_state(s)
        ss.step(4)
        got = ss.download_state()
        dts = [d.dt for d in ss.domains]
    assert np.array_equal(got, ref.state())
    assert all(dt == ref.scalars()[0] for dt in dts), (dts, ref.scalars())


@pytest.mark.parametrize("exchange,W,same", [("stage", 2, False), ("stage", 3, True), ("step", 6, False),
                                              ("step", 7, True)])
def test_oracle_slabs_overlap_bound_is_tight(oracle_lib, monkeypatch, exchange, W, same):
    """The reach is the bound: one plane less of overlap than the measured
    reach (3 per stage, 7 per step) changes the owned planes; exactly the
    reach keeps them (the defaults add a plane of margin)."""
    import freeshearlayer_b200 as fsl
    from freeshearlayer_b200 import slabs as S
    monkeypatch.setitem(S.STAGE_RADIUS, 0, min(W, S.STAGE_RADIUS[0]))
    monkeypatch.setitem(S.RADIUS, 0, min(W, S.RADIUS[0]))
    p, s = _case(oracle_lib, 1, 0)
    ref = oracle_lib.Oracle(p)
    ref.set_state(s)
    ref.step(4)
    with S.SlabSet(fsl._as_params(p), 3, overlap=W, domain_factory=OracleDomain, exchange=exchange) as ss:
        ss.upload_state(s)
        ss.step(4)
        assert np.array_equal(ss.download_state(), ref.state()) == same


def _rank_main(rank, world, port, exchange, q):
    import datetime
    import os
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import freeshearlayer_b200 as fsl
    from freeshearlayer_b200.slabs import DistributedSlab
    from oracle import oracle as orc
    from tests.test_slabs_oracle import OracleDomain, _case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p, s = _case(orc, 1, 0)
        ds = DistributedSlab(fsl._as_params(p), domain_factory=OracleDomain, exchange=exchange)
        ds.upload_state(s)
        ds.step(4)
        full = ds.gather_state(0)
        q.put((rank, ds.dom.dt, None if full is None else full.tobytes()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("exchange", ["step", "stage"])
def test_oracle_slabs_over_gloo_ranks(oracle_lib, exchange):
    """The same over two gloo ranks (DistributedSlab): point-to-point overlap
    messages and an all-reduce MAX of the Courant number."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, exchange, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    # read before joining: a rank cannot exit while its result is unread in the pipe
    res = sorted((q.get(timeout=120) for _ in range(2)), key=lambda x: x[0])
    for pr in procs:
        pr.join(60)
        assert pr.exitcode == 0
    p, s = _case(oracle_lib, 1, 0)
    ref = oracle_lib.Oracle(p)
    ref.set_state(s)
    ref.step(4)
    assert np.array_equal(np.frombuffer(res[0][2], np.float64), ref.state())
    assert res[0][1] == res[1][1] == ref.scalars()[0]
