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


def _bwd_worker(rank, world, port, ret):
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "hddm-solver-postprocessors_b200")):
        sys.path.insert(0, p)
    import hddm_b200 as H
    import oracle as O
    from hddm_b200.shard import backward_sharded, gather_outputs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    hg = H.HostGrid.adaptive(10, 1500, 8, seed=7)        # every rank builds the same grid
    gold = O.Gold(*hg.arrays())
    X = H.gen_points(10, 77, kind=2, seed=4, kink_reject=1e-6)
    C = np.random.default_rng(5).standard_normal((len(X), 8))
    lo, hi = shard_range(len(X), rank, world)

    def oracle_backward(grid, x, gout):
        gx, gs = grid.gradient(x.numpy(), gout.numpy())
        return torch.from_numpy(gx), torch.from_numpy(gs)

    gx, gs = backward_sharded(gold, torch.from_numpy(X[lo:hi]), torch.from_numpy(C[lo:hi]),
                              backward=oracle_backward)
    gx_all = gather_outputs(gx, len(X))
    if rank == 0:
        rx, rs = gold.gradient(X, C)
        ret.put((bool(np.array_equal(gx_all.numpy(), rx)),
                 float(np.abs(gs.numpy() - rs).max() / np.abs(rs).max())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharded_backward():
    """dL/dx stays per point; dL/dsurplus summed over both ranks' points by
    one all-reduce equals the whole batch's gradient (up to the order of the
    FP64 additions)."""
    ctx = mp.get_context("spawn")
    ret = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bwd_worker, args=(r, 2, port, ret)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    gx_equal, gs_rel = ret.get(timeout=10)
    assert gx_equal
    assert gs_rel <= 1e-13


def test_shard_states_assigns_every_state_once():
    from hddm_b200.shard import shard_states, state_rows
    costs = [50, 0, 70, 10, 40, 40, 5]
    for world in (1, 2, 3, 8):
        owned = shard_states(costs, world)
        assert len(owned) == world
        flat = sorted(s for o in owned for s in o)
        assert flat == list(range(len(costs)))
        assert all(o == sorted(o) for o in owned)
        assert owned == shard_states(costs, world)               # deterministic
    # largest first to the least loaded rank: 70 | 50 | 40+40 ... for 3 ranks
    loads = [sum(costs[s] for s in o) for o in shard_states(costs, 3)]
    assert max(loads) - min(loads) <= max(costs)
    assert shard_states([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard_states(costs, 0)
    counts = [3, 0, 2, 4]
    assert state_rows([2, 0], counts).tolist() == [3, 4, 0, 1, 2]
    assert state_rows([1], counts).tolist() == []


def _state_worker(rank, world, port, ret):
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "hddm-solver-postprocessors_b200")):
        sys.path.insert(0, p)
    import hddm_b200 as H
    import oracle as O
    from hddm_b200.shard import gather_state_outputs, shard_states, state_rows
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nnos = [900, 3000, 400, 1500, 2200]
    counts = [3, 0, 7, 1, 4]
    X = H.gen_points(10, sum(counts), kind=2, seed=8)
    owned = shard_states([c * n for c, n in zip(counts, nnos)], world)
    # a rank builds only the grids of its own states
    parts = []
    for s in owned[rank]:
        hg = H.HostGrid.adaptive(10, nnos[s], 12, seed=30 + s)
        parts.append(O.Gold(*hg.arrays()).interpolate(X[state_rows([s], counts)]))
    local = torch.from_numpy(np.concatenate(parts) if parts else np.zeros((0, 12)))
    full = gather_state_outputs(local, owned, counts)
    if rank == 0:
        ref = np.concatenate([O.Gold(*H.HostGrid.adaptive(10, nnos[s], 12, seed=30 + s).arrays())
                              .interpolate(X[state_rows([s], counts)]) for s in range(len(nnos))])
        ret.put((bool(np.array_equal(full.numpy(), ref)), [len(o) for o in owned]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_whole_state_sharding():
    """A multistate set split by whole states: each rank holds only its own
    states' grids, evaluates all their points, and the gathered outputs equal
    the whole batch in its own row order."""
    ctx = mp.get_context("spawn")
    ret = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_state_worker, args=(r, 2, port, ret)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    equal, per_rank = ret.get(timeout=10)
    assert equal
    assert sum(per_rank) == 5 and min(per_rank) >= 1
