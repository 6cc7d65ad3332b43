"""Point sharding across ranks (one process per GPU).

Points are independent and every rank holds the whole grid, so a batch is
split into contiguous per-rank ranges and no collective touches the forward
data path; `gather_outputs` reassembles a split batch where a caller wants it
on every rank (test and tooling use).  The backward's dL/dsurplus is a sum
over points: `backward_sharded` adds the ranks' partial sums with one
all-reduce.
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
