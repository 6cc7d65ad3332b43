"""Sharding across ranks (one process per GPU).

Points are independent and grids are read-only, so no collective touches the
forward data path.  Two ways to split a call:
* by points (`shard_range`): every rank holds every grid and takes a
  contiguous range of the batch;
* by whole states of a multistate set (`shard_states`, `state_rows`): each
  rank holds only the grids of its own states and takes all their points,
  for sets whose grids do not all fit on one GPU, or that should not be
  replicated.
`gather_outputs` and `gather_state_outputs` reassemble a split batch where a
caller wants it on every rank.  The backward's dL/dsurplus is a sum over
points: `backward_sharded` adds the ranks' partial sums with one all-reduce.
"""


def shard_range(npts, rank, world):
    """Contiguous [lo, hi) of a batch of npts points owned by `rank`; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(npts, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_outputs(local, npts, group=None):
    """All-gather per-rank output rows (torch tensors, shard_range order) into [npts, ...]."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    sizes = [shard_range(npts, r, world) for r in range(world)]
    pad = max(hi - lo for lo, hi in sizes)
    buf = torch.zeros((pad,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    buf[: local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[: hi - lo] for p, (lo, hi) in zip(parts, sizes)])


def shard_states(costs, world):
    """Whole states of a multistate set per rank: largest cost first, each to
    the least loaded rank (ties to the lower rank).  `costs[s]` is state s's
    work, e.g. its point count times its node count.  Returns, per rank, its
    state indices in increasing order; every state goes to exactly one rank."""
    if world < 1:
        raise ValueError(f"world {world} < 1")
    if any(c < 0 for c in costs):
        raise ValueError("negative state cost")
    load = [0.0] * world
    owned = [[] for _ in range(world)]
    for s in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        owned[r].append(s)
        load[r] += costs[s]
    return [sorted(o) for o in owned]


def state_rows(states, counts):
    """Row indices, in the whole batch, of the points of `states` (in the
    order given), where state s owns counts[s] consecutive rows."""
    import numpy as np
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    if len(states) == 0:
        return np.zeros(0, np.int64)
    return np.concatenate([np.arange(off[s], off[s + 1], dtype=np.int64) for s in states])


def gather_state_outputs(local, owned, counts, group=None):
    """All-gather per-rank outputs of whole states (rank r's rows are those of
    owned[r], in state_rows order) into the whole batch's row order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if len(owned) != world:
        raise ValueError(f"{len(owned)} state lists for {world} ranks")
    sizes = [int(sum(counts[s] for s in o)) for o in owned]
    pad = max(sizes + [1])
    buf = torch.zeros((pad,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    buf[: local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = torch.empty((int(sum(counts)),) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r in range(world):
        rows = torch.from_numpy(state_rows(owned[r], counts)).to(local.device)
        out[rows] = parts[r][: sizes[r]]
    return out


def backward_sharded(grid, x_local, gout_local, group=None, backward=None):
    """Backward over a point batch split across ranks (one process per GPU).

    Each rank passes its own shard (shard_range order) of the points and of
    dL/dvalue.  dL/dx is point-local and stays on the rank; dL/dsurplus is a
    sum over all points, so the per-rank sums are added with one all-reduce
    (NCCL on GPUs) and every rank returns the whole batch's gradient.  With
    one rank this is the plain backward.  `backward(grid, x, gout)` returns
    (gx, gsurplus) tensors; it defaults to hddm_b200.backward, the GPU kernel.
    """
    import torch.distributed as dist
    if backward is None:
        from . import backward as backward  # the GPU kernel
    gx, gs = backward(grid, x_local, gout_local)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(gs, op=dist.ReduceOp.SUM, group=group)
    return gx, gs
