"""Point sharding across ranks (one process per GPU).

Points are independent and every rank holds the whole grid, so a batch is
split into contiguous per-rank ranges and no collective touches the data
path; `gather_outputs` reassembles a split batch where a caller wants it on
every rank (test and tooling use).
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
