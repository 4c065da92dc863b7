"""The bench's multi-rank host logic on CPU: two gloo ranks, each timing its
own replica, agree on the slowest rank's time and the whole-job rate; the
reference arm does its work on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms_local = [12.5, 20.0][rank]
        ms = bench.max_over_ranks(torch, dist, ms_local, device="cpu")
        rate = bench.whole_job_rate(1000, world, ms)
        # the reference arm: ranks other than 0 return without work or output
        buf = io.StringIO()
        args = type("A", (), {"grid": "8x8x8", "steps": 1, "warmup": 0})()
        if rank != 0:
            with redirect_stdout(buf):
                bench.main_reference(args)
        dist.barrier()
        q.put((rank, ms, rate, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    # read before joining: a rank cannot exit while its result is unread in the pipe
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, ms, rate, out in res:
        assert ms == 20.0                       # the slowest rank's time on every rank
        assert rate == pytest.approx(1000 * 2 / 0.020)
        if rank != 0:
            assert out == ""
