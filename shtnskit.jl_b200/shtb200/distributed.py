"""Field sharding across ranks (one process per GPU, ``torch.distributed``).

Batched transforms are independent per field, so a batch splits into contiguous field
ranges with no collective in the transforms themselves (the multi-GPU mode of the
reference's batch API, src/batch_transforms.jl; its transpose-based distributed plans are
a different path). ``synthesis_batch_sharded`` / ``analysis_batch_sharded`` run a batch that
way and, on request, all-gather the shards so that every rank holds the whole result; the
other collectives appear only around timing: a barrier before and after a timed region
and the maximum of the per-rank times.
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


def gather_fields(local: torch.Tensor, n_total: int) -> torch.Tensor:
    """Every rank's field shard (trailing index of a column-major batch, shards in rank order as
    ``shard_range`` cuts them) concatenated into the whole batch, on every rank.

    The shards go through one ``all_gather_into_tensor`` (NCCL on GPUs, gloo on CPUs) padded to
    the largest shard, since the collective moves equal sizes; complex values travel as pairs of
    reals. Without an initialized process group the local batch is returned as it is.
    """
    rank, w = world()
    if w == 1:
        return local
    per = shard_range(n_total, 0, w)[1]            # the largest shard (rank 0 gets the remainder first)
    nloc = local.shape[-1]
    lead = tuple(local.shape[:-1])
    elems = 1
    for d in lead:
        elems *= d
    flat = local.permute(*reversed(range(local.dim()))).reshape(nloc, elems)   # [field][element]
    if flat.is_complex():
        flat = torch.view_as_real(flat).reshape(nloc, 2 * elems)
    buf = torch.zeros((per, flat.shape[1]), dtype=flat.dtype, device=flat.device)
    buf[:nloc] = flat
    out = torch.empty((w * per, flat.shape[1]), dtype=flat.dtype, device=flat.device)
    dist.all_gather_into_tensor(out, buf)
    parts = [out[r * per: r * per + (shard_range(n_total, r, w)[1] - shard_range(n_total, r, w)[0])]
             for r in range(w)]
    full = torch.cat(parts, dim=0)
    if local.is_complex():
        full = torch.view_as_complex(full.reshape(n_total, elems, 2).contiguous())
    # back to the column-major (..., n_total) view of a [field][...] buffer
    return full.reshape((n_total,) + lead[::-1]).permute(*reversed(range(len(lead) + 1)))


def sharded(transform, cfg, x, *, gather: bool = True, **kwargs):
    """A batched transform run field-sharded: every rank passes the whole batch ``x``, transforms
    its own contiguous field range on its own GPU (``transform(cfg, shard, **kwargs)``, no
    collective), and with ``gather`` all ranks receive the whole result (one all-gather);
    without it each rank returns its shard."""
    mine = shard_fields(x)
    if mine.shape[-1] == 0 and x.shape[-1] > 0:
        # fewer fields than ranks: this rank's shard is empty; a one-field call gives the
        # output's shape, of which it keeps no field
        out = transform(cfg, x[..., :1], **kwargs)[..., :0]
    else:
        out = transform(cfg, mine, **kwargs)
    return gather_fields(out, x.shape[-1]) if gather else out


def synthesis_batch_sharded(cfg, alm, *, gather: bool = True, **kwargs):
    """``synthesis_batch`` with the fields split over the ranks of the process group."""
    from .transforms import synthesis_batch
    return sharded(synthesis_batch, cfg, alm, gather=gather, **kwargs)


def analysis_batch_sharded(cfg, f, *, gather: bool = True, **kwargs):
    """``analysis_batch`` with the fields split over the ranks of the process group."""
    from .transforms import analysis_batch
    return sharded(analysis_batch, cfg, f, gather=gather, **kwargs)
