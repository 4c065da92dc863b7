"""x-slab decomposition of one domain over several contexts (one per GPU).

The reference's distributed variant (src-par/mpi_layer2.c:135-254) splits the
domain into x-slabs, one per MPI rank, and exchanges one ghost plane of U, of
the face states and of mu_SGS with blocking sends in every stage
(src-par/boundCondInGhostCells.c:23-102, src-par/boundCondOnInterfaces.c:20-99,
src-par/communication.c:6-93), with an MPI_Allreduce MAX of the Courant number
(src-par/helpers.c:44).

Here a slab is a whole domain context whose x-extent is its owned planes plus
W overlap planes on each side.  A step changes a plane only through planes
within RADIUS of it (per stage two planes for the reference reconstruction,
three for PPM, and the SGS viscosity's reach once per step), so after one
step the planes within W of a slab's ends may be wrong (they saw the slab's
own x-boundary) while every owned plane is exactly what the undivided domain
computes.  In the x-periodic temporal setup the undivided domain is not
translation-invariant: its ghost planes wrap, but the SGS test filter keeps
the zero bands of a domain boundary at the seam between planes LEN and 1.  A
slab whose overlap crosses the seam therefore lists its planes in ascending
global order, which puts the seam on its own periodic boundary and the
discontinuity between unrelated planes inside its overlap.  Once per step
each slab's overlap planes are refreshed from its neighbours' owned planes,
and before each step the Courant maximum over the owned planes is combined by
a maximum across slabs, so that every slab rescales deltaT to the same value.
One exchange per step instead of one per stage, at the price of 2W extra
planes of work per slab.

exchange="stage" refreshes the overlap after every stage instead, as the
reference does: the stage state of every local plane is then exact when the
next stage starts, so W need only cover one stage's reach (STAGE_RADIUS), half
the redundant work for three exchanges per step.

`SlabSet` drives several slabs from one process (one device, or one device
per slab); `DistributedSlab` drives one slab per rank of a torch.distributed
process group (NCCL: device buffers; gloo: host buffers).
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

import numpy as np

# Overlap widths, at least the x-reach of one step in planes: three stages of
# 2 (reference reconstruction) or 3 (PPM) plus the SGS viscosity's reach into
# the first stage.  Measured by perturbing one plane: 7 for the reference
# reconstruction and 9 for PPM; the defaults keep a plane of margin.
RADIUS = {0: 8, 1: 10}

# Overlap widths for an exchange after every stage: one stage reaches 2
# planes (reference reconstruction) or 3 (PPM) through the x-stencil, and
# every stage reads the step's SGS viscosity at the neighbouring planes, whose
# own reach into U^n is 2 (velocities, the test filter and the strain), so 3
# for the first stage.  Measured by perturbing one plane: 3 and 2 for stages 1
# and 2 with the reference reconstruction, 3 and 3 with PPM; the defaults keep
# a plane of margin.
STAGE_RADIUS = {0: 4, 1: 4}
EXCHANGES = ("step", "stage")


@dataclass(frozen=True)
class Slab:
    """Owned global planes a..b (1-based) of a domain of LEN planes, W
    overlap planes before (wl) and after (wr) them, and whether x is periodic.

    The local domain holds the owned and overlap planes in ascending global
    order.  When the overlap wraps across the periodic seam (between planes
    LEN and 1), this puts the seam on the local domain's own periodic
    boundary, where the undivided domain has it (its ghost fill wraps there,
    while the SGS test filter keeps the zero bands of a domain boundary), and
    puts the discontinuity between unrelated planes (the junction) inside the
    overlap, which is refreshed every step."""
    index: int
    a: int
    b: int
    wl: int
    wr: int
    LEN: int

    @property
    def n(self) -> int:
        return self.b - self.a + 1

    @property
    def local_len(self) -> int:
        return self.n + self.wl + self.wr

    def global_planes(self) -> np.ndarray:
        """Global plane (1-based) held in each local plane 1..local_len."""
        g = (np.arange(self.a - self.wl, self.b + self.wr + 1) - 1) % self.LEN + 1
        return np.sort(g)

    @property
    def own0(self) -> int:
        """Local index of the first owned plane (owned planes are contiguous)."""
        return self.local_index(self.a)

    @property
    def own1(self) -> int:
        return self.own0 + self.n - 1

    def local_index(self, g: int) -> int:
        """Local plane (1-based) holding global plane g."""
        return int(np.nonzero(self.global_planes() == g)[0][0]) + 1


def layout(LEN: int, nslabs: int, overlap: int, periodic: bool) -> list[Slab]:
    """Split planes 1..LEN into nslabs contiguous slabs (sizes differing by at
    most one).  A periodic domain gives every slab overlap on both sides; a
    non-periodic one gives none before the first and none after the last.
    Each slab must own at least `overlap` planes, and a slab with its overlap
    must not cover the domain twice."""
    if nslabs < 1 or LEN < nslabs:
        raise ValueError("layout: %d planes do not split into %d slabs" % (LEN, nslabs))
    if nslabs == 1:
        return [Slab(0, 1, LEN, 0, 0, LEN)]
    base, extra = divmod(LEN, nslabs)
    if base < overlap:
        raise ValueError("layout: slabs of %d planes are thinner than the overlap %d" % (base, overlap))
    out, a = [], 1
    for r in range(nslabs):
        n = base + (r < extra)
        wl = overlap if (periodic or r > 0) else 0
        wr = overlap if (periodic or r < nslabs - 1) else 0
        if n + wl + wr > LEN:
            raise ValueError("layout: a slab of %d planes with its overlap covers the %d planes more than once"
                             % (n, LEN))
        out.append(Slab(r, a, a + n - 1, wl, wr, LEN))
        a += n
    return out


def slab_params(p, slab: Slab):
    q = copy.copy(p)
    q.LEN = slab.local_len
    return q


def owner(slabs: list[Slab], g: int) -> Slab:
    for s in slabs:
        if s.a <= g <= s.b:
            return s
    raise ValueError("plane %d is owned by no slab" % g)


def exchange_plan(slabs: list[Slab]):
    """The copies of one exchange, in one order for every caller: (src slab,
    src local plane, dst slab, dst local plane, n) -- each overlap plane of a
    slab from the slab that owns it, runs of consecutive planes merged."""
    plan = []
    for s in slabs:
        gp = s.global_planes()
        for q in range(s.local_len):
            g = int(gp[q])
            if s.a <= g <= s.b:
                continue
            o = owner(slabs, g)
            i = o.local_index(g)
            if plan:
                src, i0, dst, j0, n = plan[-1]
                if src == o.index and dst == s.index and i == i0 + n and q + 1 == j0 + n:
                    plan[-1] = (src, i0, dst, j0, n + 1)
                    continue
            plan.append((o.index, i, s.index, q + 1, 1))
    return plan


def _check_overlap(p, overlap, exchange="step"):
    if exchange not in EXCHANGES:
        raise ValueError("exchange: 'step' or 'stage'")
    if exchange == "stage" and p.nStages != 3:
        raise ValueError("exchange='stage' steps the fused RK3 stages (nStages = 3)")
    need = (RADIUS if exchange == "step" else STAGE_RADIUS)[p.recon]
    W = need if overlap is None else int(overlap)
    if W < need:
        raise ValueError("overlap %d below the %s's reach of %d planes" % (W, exchange, need))
    return W


def _check_phased(exchange, phased):
    if phased and exchange == "stage":
        raise ValueError("exchange='stage' runs the fused stages (fsl_step_stage)")


class SlabSet:
    """Several x-slabs of one domain driven from one process.

    devices: one CUDA device index per slab (default: all on the current
    device).  staging "host" moves overlap planes through numpy arrays;
    "device" through CUDA tensors (peer copies between devices) and combines
    the Courant maximum in device memory.  With device staging on one device
    the exchange and the combination are ordered between the slabs' streams
    by CUDA events, without waiting on the host, so the slabs' kernels may
    also overlap one another.

    exchange "step" refreshes the overlap planes once per step, "stage"
    after every stage (a narrower default overlap).  domain_factory(params)
    makes each slab's context (default: Domain)."""

    def __init__(self, params, nslabs: int, overlap: int | None = None, devices=None,
                 staging: str = "host", domain_factory=None, exchange: str = "step"):
        from . import Domain, SETUP_TEMPORAL, _as_params
        p = _as_params(params)
        self.p = p
        self.W = _check_overlap(p, overlap, exchange)
        self.exchange_mode = exchange
        self.slabs = layout(p.LEN, nslabs, self.W, p.setup == SETUP_TEMPORAL)
        self.plan = exchange_plan(self.slabs)
        if staging not in ("host", "device"):
            raise ValueError("staging: 'host' or 'device'")
        self.staging = staging
        self.devices = list(devices) if devices is not None else None
        self.domains = []
        for s in self.slabs:
            with self._on(s.index):
                d = (domain_factory or Domain)(slab_params(p, s))
                d.set_courant_range(s.own0, s.own1)
                self.domains.append(d)
        self.plane = p.HIG * 5 * p.DEP
        self._bufs = {}
        self._read = {}     # per buffer: the event after the set that last read it
        self._ordered = staging == "device" and self.devices is None

    def _stream(self, r):
        import torch
        return torch.cuda.ExternalStream(self.domains[r].stream)

    def _on(self, r):
        import contextlib
        if self.devices is None:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.device(self.devices[r])

    def close(self):
        for d in self.domains:
            d.close()       # waits for the slab's stream, which may still read a buffer
        self.domains = []
        self._bufs, self._read = {}, {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- state ------------------------------------------------------------------
    def upload_state(self, state: np.ndarray):
        """The undivided U^n ([LEN][HIG][5][DEP]) into the slabs, overlaps included."""
        u = np.asarray(state, np.float64).reshape(self.p.LEN, self.plane)
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                d.upload_state(np.ascontiguousarray(u[s.global_planes() - 1]))

    def download_state(self) -> np.ndarray:
        """The owned planes of every slab, as the undivided U^n."""
        out = np.empty((self.p.LEN, self.plane), np.float64)
        for s, d in zip(self.slabs, self.domains):
            buf = np.empty(s.n * self.plane, np.float64)
            with self._on(s.index):
                d.get_planes(s.own0, s.n, buf)
            out[s.a - 1:s.b] = buf.reshape(s.n, self.plane)
        return out.reshape(-1)

    # --- one step -----------------------------------------------------------------
    def combine_courant(self):
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                d.courant_prepare()
        if self._ordered:
            self._combine_courant_ordered()
            return
        if self.staging == "device":
            self._combine_courant_device()
            return
        m = 0.0
        for d in self.domains:
            c = d.get_courant_max()
            m = c if c > m else m
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                d.set_courant_max(m)

    def _combine_courant_device(self):
        import torch
        ts = []
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                d.sync()
                ts.append(device_scalar(d.courant_bits_ptr(), torch.cuda.current_device()))
        # non-negative doubles order like their bit patterns (as int64)
        m = ts[0].clone()
        for t in ts[1:]:
            m = torch.maximum(m, t.to(m.device))
        for t in ts:
            t.copy_(m.to(t.device))
        torch.cuda.synchronize()

    def _combine_courant_ordered(self):
        """The maximum of the slabs' device scalars on the current stream,
        after each slab's stream has produced its scalar and before any slab
        stream reads the result."""
        import torch
        cur = torch.cuda.current_stream()
        ts = []
        for r, d in enumerate(self.domains):
            ts.append(device_scalar(d.courant_bits_ptr(), torch.cuda.current_device()))
            ev = torch.cuda.Event()
            ev.record(self._stream(r))
            cur.wait_event(ev)
        # non-negative doubles order like their bit patterns (as int64)
        m = ts[0].clone()
        for t in ts[1:]:
            m = torch.maximum(m, t)
        for t in ts:
            t.copy_(m)
        done = torch.cuda.Event()
        done.record(cur)
        for r in range(len(self.domains)):
            self._stream(r).wait_event(done)

    def _exchange_ordered(self):
        """Each overlap run: the owner's stream gathers it into a device
        buffer, the receiver's stream waits for that and scatters it; the next
        gather into the same buffer waits for the scatter that read it."""
        import torch
        for src, i0, dst, j0, n in self.plan:
            key = (src, dst, i0, n)
            buf = self._buffer(src, dst, i0, n)
            ss, ds = self._stream(src), self._stream(dst)
            if key in self._read:
                ss.wait_event(self._read[key])
            self.domains[src].get_planes_async(i0, n, buf)
            filled = torch.cuda.Event()
            filled.record(ss)
            ds.wait_event(filled)
            self.domains[dst].set_planes_async(j0, n, buf)
            read = torch.cuda.Event()
            read.record(ds)
            self._read[key] = read

    def exchange(self):
        if not self.plan:
            return
        if self._ordered:
            self._exchange_ordered()
            return
        staged = []
        for src, i0, dst, j0, n in self.plan:
            with self._on(src):
                buf = self._buffer(src, dst, i0, n)
                self.domains[src].get_planes(i0, n, buf)
            staged.append((buf, dst, j0, n))
        if self.staging == "device":
            import torch
            torch.cuda.synchronize()
        for buf, dst, j0, n in staged:
            with self._on(dst):
                if self.staging == "device" and self.devices is not None:
                    buf = buf.to("cuda:%d" % self.devices[dst])
                self.domains[dst].set_planes(j0, n, buf)

    def _buffer(self, src, dst, i0, n):
        key = (src, dst, i0, n)
        if key not in self._bufs:
            if self.staging == "device":
                import torch
                self._bufs[key] = torch.empty(n * self.plane, dtype=torch.float64, device="cuda")
            else:
                self._bufs[key] = np.empty(n * self.plane, np.float64)
        return self._bufs[key]

    def step(self, n: int = 1, phased: bool = False):
        _check_phased(self.exchange_mode, phased)
        for _ in range(n):
            self.combine_courant()
            if self.exchange_mode == "stage":
                for _stage in range(3):
                    for s, d in zip(self.slabs, self.domains):
                        with self._on(s.index):
                            d.step_stage()
                    self.exchange()
                continue
            for s, d in zip(self.slabs, self.domains):
                with self._on(s.index):
                    d.step_phased(1) if phased else d.step(1)
            self.exchange()

    def sync(self):
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                d.sync()

    # --- integrals over the whole domain ---------------------------------------------
    def sums(self) -> np.ndarray:
        """Volume integrals of the conserved variables: each slab's over its
        owned planes, added (slab order; equal to the undivided domain's to
        rounding)."""
        out = None
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                x = d.sums()
            out = x if out is None else out + x
        return out

    def plane_sums(self) -> np.ndarray:
        """Per y-row sums over the owned x-z planes, added across slabs."""
        out = None
        for s, d in zip(self.slabs, self.domains):
            with self._on(s.index):
                x = d.plane_sums()
            out = x if out is None else out + x
        return out


def device_scalar(ptr: int, device: int):
    """A one-element int64 CUDA tensor over device memory at `ptr` (not owned)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (1,), "typestr": "<i8", "data": (ptr, False), "version": 3,
                                    "strides": None}

    return torch.as_tensor(_View(), device="cuda:%d" % device)


class DistributedSlab:
    """This rank's slab of a domain split over the ranks of a torch.distributed
    process group (one rank per GPU).  With NCCL the overlap planes travel in
    CUDA tensors; with gloo in host tensors.  Every rank takes the same
    collective steps in the same order.

    exchange: "step" or "stage", as for SlabSet.  domain_factory(params)
    makes the slab's context (default: Domain on the current CUDA device)."""

    def __init__(self, params, group=None, overlap: int | None = None, domain_factory=None,
                 exchange: str = "step"):
        import torch
        import torch.distributed as dist
        from . import Domain, SETUP_TEMPORAL, _as_params
        p = _as_params(params)
        self.p, self.group = p, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.W = _check_overlap(p, overlap, exchange)
        self.exchange_mode = exchange
        self.slabs = layout(p.LEN, self.size, self.W, p.setup == SETUP_TEMPORAL)
        self.slab = self.slabs[self.rank]
        self.on_device = dist.get_backend(group) == "nccl"
        factory = domain_factory or Domain
        self.dom = factory(slab_params(p, self.slab))
        self.dom.set_courant_range(self.slab.own0, self.slab.own1)
        self.plane = p.HIG * 5 * p.DEP
        dev = "cuda" if self.on_device else "cpu"
        # this rank's part of the exchange, in the plan's order (the same on
        # every rank): per neighbour pair the messages are issued in one
        # order, so that they match by order where tags are not kept (NCCL)
        self.plan = [(t, e) for t, e in enumerate(exchange_plan(self.slabs)) if self.rank in (e[0], e[2])]
        self._bufs = {t: torch.empty(e[4] * self.plane, dtype=torch.float64, device=dev) for t, e in self.plan}

    def _buf(self, t):
        return t if self.on_device else t.numpy()

    def _global(self, r):
        import torch.distributed as dist
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def close(self):
        self.dom.close()

    # --- state ------------------------------------------------------------------
    def upload_state(self, state: np.ndarray):
        """Each rank passes the undivided U^n and keeps its planes."""
        u = np.asarray(state, np.float64).reshape(self.p.LEN, self.plane)
        self.dom.upload_state(np.ascontiguousarray(u[self.slab.global_planes() - 1]))

    def gather_state(self, dst: int = 0):
        """The undivided U^n on rank `dst` (None elsewhere)."""
        import torch
        import torch.distributed as dist
        s = self.slab
        nmax = max(x.n for x in self.slabs)
        dev = "cuda" if self.on_device else "cpu"
        mine = torch.zeros(nmax * self.plane, dtype=torch.float64, device=dev)
        self.dom.get_planes(s.own0, s.n, self._buf(mine))
        parts = [torch.empty_like(mine) for _ in range(self.size)] if self.rank == dst else None
        dist.gather(mine, parts, dst=self._global(dst), group=self.group)
        if self.rank != dst:
            return None
        out = np.empty((self.p.LEN, self.plane), np.float64)
        for x, t in zip(self.slabs, parts):
            out[x.a - 1:x.b] = t.cpu().numpy()[:x.n * self.plane].reshape(x.n, self.plane)
        return out.reshape(-1)

    # --- one step -----------------------------------------------------------------
    def _sum_all(self, x: np.ndarray) -> np.ndarray:
        import torch
        import torch.distributed as dist
        t = torch.from_numpy(np.ascontiguousarray(x, np.float64).ravel())
        if self.on_device:
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy().reshape(np.shape(x))

    def sums(self) -> np.ndarray:
        """Volume integrals of the conserved variables over the whole domain:
        the owned planes' integrals, all-reduced with SUM on every rank."""
        return self._sum_all(self.dom.sums())

    def plane_sums(self) -> np.ndarray:
        """Per y-row sums over all x-z planes, all-reduced with SUM."""
        return self._sum_all(self.dom.plane_sums())

    def combine_courant(self):
        """The owned Courant maximum, combined by an all-reduce MAX
        (src-par/helpers.c:44)."""
        import torch
        import torch.distributed as dist
        self.dom.courant_prepare()
        m = self.dom.get_courant_max()
        t = torch.tensor([m], dtype=torch.float64, device="cuda" if self.on_device else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        self.dom.set_courant_max(float(t.item()))

    def exchange(self):
        """Overlap planes from the slabs that own them, as point-to-point
        messages (the per-stage sends of src-par/boundCondInGhostCells.c:60-73,
        one set per step or per stage)."""
        import torch
        import torch.distributed as dist
        if not self.plan:
            return
        ops = []
        for t, (src, i0, dst, j0, n) in self.plan:
            buf = self._bufs[t]
            if src == self.rank:
                self.dom.get_planes(i0, n, self._buf(buf))
                ops.append(dist.P2POp(dist.isend, buf, self._global(dst), self.group, tag=t))
            else:
                ops.append(dist.P2POp(dist.irecv, buf, self._global(src), self.group, tag=t))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        if self.on_device:
            torch.cuda.current_stream().synchronize()
        for t, (src, i0, dst, j0, n) in self.plan:
            if dst == self.rank:
                self.dom.set_planes(j0, n, self._buf(self._bufs[t]))

    def step(self, n: int = 1, phased: bool = False):
        _check_phased(self.exchange_mode, phased)
        for _ in range(n):
            self.combine_courant()
            if self.exchange_mode == "stage":
                for _stage in range(3):
                    self.dom.step_stage()
                    self.exchange()
                continue
            self.dom.step_phased(1) if phased else self.dom.step(1)
            self.exchange()
