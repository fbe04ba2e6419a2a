"""bench.py --gpus N runs N independent replicas (the path does not shard on one
job): the whole-job rate is all ranks' points over the slowest rank's time.  The
reduction runs here on two gloo ranks over 127.0.0.1."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [40.0, 50.0][rank]  # rank 1 is the slow one
        rate, total_ms = bench.whole_job_rate(1_000_000, 5, local_ms, world)
        out.put((rank, rate, total_ms))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, rate, total_ms in res:
        assert total_ms == pytest.approx(50.0)
        assert rate == pytest.approx(2 * 1_000_000 * 5 / 0.050)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    rate, total_ms = bench.whole_job_rate(10, 2, 4.0, 1)
    assert (rate, total_ms) == (10 * 2 / 0.004, 4.0)
