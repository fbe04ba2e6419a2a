"""The sharded form (nextdbscan-exa_b200/sharded.py): spatial slabs with a 2r halo,
one local run per rank, the merge of components across slab boundaries and the
border pass with the merged ids.  Its outputs must equal one run over the whole
input (the reference's multi-rank results, data_process.cpp:129-233, are those of
the single-rank run).

On the CPU the ranks are gloo processes over 127.0.0.1 whose local step is the
oracle (cell restatement plus the border rule with given ids); on the GPU two gloo
ranks share cuda:0 and run the library itself.  The ranks' kernels never wait on
one another: every exchange is a host-side collective between the local runs."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def workload(name):
    sys.path.insert(0, ROOT)
    import importlib
    pkg = importlib.import_module("nextdbscan-exa_b200")
    if name == "c1":
        w = pkg.synthetic.config1(n=24_000)
    elif name == "c2":
        w = pkg.synthetic.config2(n=40_000)
        w = type(w)(w.name, w.coords, w.eps * 6, w.min_pts)  # denser: clusters that cross the slabs
    elif name == "c3":
        w = pkg.synthetic.config3(n=9_000)
    elif name == "c5":
        w = pkg.synthetic.config5(n=30_000)
    else:  # special points stay on their own ranks; minPts <= 0 makes each one a cluster
        rng = np.random.default_rng(5)
        x = rng.normal(0, 1.0, (6_000, 2)).astype(np.float32)
        x[::97, 0] = np.nan
        x[::89, 1] = np.inf
        x[::83, 0] = np.finfo(np.float32).max
        return x, 0.15, 0
    return w.coords, w.eps, w.min_pts


def _rank(rank, world, port, name, use_gpu, full, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import importlib
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        pkg = importlib.import_module("nextdbscan-exa_b200")
        sharded = importlib.import_module("nextdbscan-exa_b200.sharded")
        x, eps, m = workload(name)
        cuts = np.linspace(0, x.shape[0], world + 1).astype(int)
        cuts[1:-1] += np.arange(1, world) * 37  # uneven blocks
        block = x[cuts[rank]:cuts[rank + 1]]
        if use_gpu:
            ctx = pkg.Context(0)
            local = sharded.gpu_local_step(ctx)
        else:
            import oracle

            def local(lx, e, mp_, full_count):
                nn, ci, _ = oracle.cells(lx, e, mp_, early=not full_count)
                return sharded.LocalResult(nn, ci, lambda ids: oracle.border_ids(lx, e, mp_, nn, ids))
        r = sharded.run_sharded(block, eps, m, local=local, full_count=full)
        q.put((rank, int(cuts[rank]), r.nn, r.cluster_index, (r.clusters, r.noise, r.core_count, r.n)))
        dist.barrier()
        if use_gpu:
            ctx.close()
    finally:
        dist.destroy_process_group()


def run_ranks(world, name, use_gpu=False, full=True):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, use_gpu, full, q)) for r in range(world)]
    for p in procs:
        p.start()
    import queue
    import time
    outs, t0 = [], time.time()
    while len(outs) < world:  # fail fast when a rank dies instead of waiting out the queue
        try:
            outs.append(q.get(timeout=2))
        except queue.Empty:
            dead = [p.exitcode for p in procs if p.exitcode not in (None, 0)]
            assert not dead, f"a rank exited with {dead}"
            assert time.time() - t0 < 300, "ranks did not report within 300 s"
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    outs.sort()
    nn = np.concatenate([o[2] for o in outs])
    ci = np.concatenate([o[3] for o in outs])
    metas = {o[4] for o in outs}
    assert len(metas) == 1, metas  # every rank reports the same global meta
    return nn, ci, metas.pop()


@pytest.mark.parametrize("world,name", [(2, "c1"), (4, "c1"), (2, "c2"), (3, "c3"), (4, "c5"), (2, "special")])
def test_sharded_equals_one_run(world, name):
    import oracle
    x, eps, m = workload(name)
    nn_o, ci_o, meta = oracle.cells(x, eps, m)
    nn, ci, (clusters, noise, cores, n) = run_ranks(world, name)
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(ci, ci_o)
    assert (clusters, noise, cores, n) == (meta["clusters"], meta["noise"], meta["cores"], meta["n"])


def test_merge_of_pairs_takes_the_smallest_index():
    sys.path.insert(0, ROOT)
    import importlib
    sharded = importlib.import_module("nextdbscan-exa_b200.sharded")
    pairs = np.array([[10, 4], [4, 4], [7, 10], [20, 15], [15, 15], [99, 99]], np.int64)
    root = sharded._merge_roots(pairs)
    assert root == {4: 4, 7: 4, 10: 4, 15: 15, 20: 15, 99: 99}
    assert sharded.reach(1.5) > 1.5 and sharded.reach(0.0) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name,full", [("c1", True), ("c2", False), ("c3", True)])
def test_sharded_on_the_gpu_equals_one_run(name, full):
    """Two ranks, each running the library on cuda:0 for its slab and halo, then
    the border pass with the merged ids (ndb_b200_assign_border)."""
    sys.path.insert(0, ROOT)
    import importlib
    pkg = importlib.import_module("nextdbscan-exa_b200")
    x, eps, m = workload(name)
    with pkg.Context(0) as ctx:
        nn_1, ci_1, res = ctx.run(x, eps, m, full_count=full)
    nn, ci, (clusters, noise, cores, n) = run_ranks(2, name, use_gpu=True, full=full)
    np.testing.assert_array_equal(ci, ci_1)
    if full:
        np.testing.assert_array_equal(nn, nn_1)
    else:
        below = nn_1 < m
        np.testing.assert_array_equal(nn[below], nn_1[below])
        np.testing.assert_array_equal(nn >= m, nn_1 >= m)
    assert (clusters, noise, cores, n) == (res.clusters, res.noise, res.core_count, res.n)
