"""Field sharding across ranks (one process per GPU, ``torch.distributed``).

Batched transforms are independent per field, so a batch splits into contiguous field
ranges with no collective in the data path (the multi-GPU mode of the reference's
batch API, src/batch_transforms.jl; its transpose-based distributed plans are a
different path). Collectives appear only around timing: a barrier before and after a
timed region and the maximum of the per-rank times.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced [start, stop) of n items for rank (the first n % world ranks get one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def world() -> tuple[int, int]:
    """(rank, world size), (0, 1) when torch.distributed is not initialized."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def barrier() -> None:
    if world()[1] > 1:
        dist.barrier()


def max_over_ranks(value: float, device: torch.device | None = None) -> float:
    """The maximum of a per-rank scalar (device time of a timed region) over all ranks."""
    if world()[1] == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_fields(x, rank: int | None = None, world_size: int | None = None):
    """This rank's slice of a batch along its trailing field index."""
    r, w = world()
    r = r if rank is None else rank
    w = w if world_size is None else world_size
    a, b = shard_range(x.shape[-1], r, w)
    return x[..., a:b]
