"""Field sharding over GPUs.

Fields (radial shells, batch members) are independent, so N processes, one per
GPU, each transform a contiguous slice of the fields with no communication on
the data path.  These helpers give the slice of a rank and, when a caller
wants the whole result on every rank, gather the slices with torch.distributed.
"""


def field_shard(nfields, rank, world):
    """Contiguous slice of `nfields` owned by `rank` (sizes differ by at most 1)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("invalid rank/world")
    base, extra = divmod(nfields, world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return slice(start, stop)


def gather_fields(local, nfields, group=None):
    """All-gather per-rank field slices (leading dimension) into the full
    [nfields, ...] tensor on every rank (uneven slices are padded for the
    collective and trimmed afterwards)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    per = -(-nfields // world)
    pad = torch.zeros((per,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    out = [parts[r][: field_shard(nfields, r, world).stop - field_shard(nfields, r, world).start]
           for r in range(world)]
    return torch.cat(out, dim=0)
