"""Multi-process path on CPU: two gloo ranks split a batch with shard_range,
each evaluates its shard (the oracle stands in for the GPU kernel here), and the
gathered result equals the whole batch; the max-over-ranks timing reduction
is the one bench.py uses."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hddm_b200.shard import shard_range


def test_shard_range_covers_batch():
    for npts in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            rs = [shard_range(npts, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == npts
            assert all(rs[k][1] == rs[k + 1][0] for k in range(world - 1))
            sizes = [hi - lo for lo, hi in rs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, ret):
    import sys
    import time
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "hddm-solver-postprocessors_b200")):
        sys.path.insert(0, p)
    import hddm_b200 as H
    import oracle as O
    from hddm_b200.shard import gather_outputs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    hg = H.HostGrid.adaptive(12, 2000, 16, seed=5)       # every rank builds the same grid
    X = H.gen_points(12, 101, kind=2, seed=3)
    lo, hi = shard_range(len(X), rank, world)
    t = time.perf_counter()
    local = torch.from_numpy(O.Gold(*hg.arrays()).interpolate(X[lo:hi]))
    dt = torch.tensor([time.perf_counter() - t], dtype=torch.float64)
    full = gather_outputs(local, len(X))
    dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    if rank == 0:
        ref = O.Gold(*hg.arrays()).interpolate(X)
        ret.put((bool(np.array_equal(full.numpy(), ref)), float(dt.item()) > 0))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_shard_and_gather():
    ctx = mp.get_context("spawn")
    ret = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ret)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    equal, timed = ret.get(timeout=10)
    assert equal and timed
