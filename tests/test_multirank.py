"""CPU, two ranks over gloo: the field-sharding host logic of the multi-GPU batch mode.

Each rank transforms its contiguous field range (the oracle stands in for the device
kernels, which are per-field independent); gathering the shards must reproduce the
single-process batch exactly, and the timing reduction must return the maximum over
ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from shtb200.distributed import barrier, max_over_ranks, shard_fields, shard_range
from oracle import sht_oracle as so

from _util import rand_alm


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nf, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = so.create_gauss_config(15, 16)
        a = rand_alm(15, 15, nf, seed=21)
        mine = shard_fields(a)
        f = so.synthesis_batch(cfg, mine) if mine.shape[-1] else np.zeros((16, cfg.nlon, 0))
        shards = [None] * world
        dist.all_gather_object(shards, f)
        t = max_over_ranks(0.5 + rank)
        barrier()
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), np.concatenate(shards, axis=2))
            np.save(os.path.join(out_dir, "tmax.npy"), np.array([t]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nf", [(2, 7), (2, 1)])
def test_two_rank_field_sharding(tmp_path, world, nf):
    mp.start_processes(_rank_main, args=(world, _free_port(), nf, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    cfg = so.create_gauss_config(15, 16)
    ref = so.synthesis_batch(cfg, rand_alm(15, 15, nf, seed=21))
    got = np.load(tmp_path / "gathered.npy")
    assert got.shape == ref.shape and np.array_equal(got, ref)
    assert float(np.load(tmp_path / "tmax.npy")[0]) == 0.5 + (world - 1)


def test_shard_range_partitions():
    for n in (0, 1, 5, 64, 65):
        for w in (1, 2, 3, 8):
            spans = [shard_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(w - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def _oracle_batch(op):
    """A batched transform on CPU torch tensors in column-major layout, the oracle standing in
    for the device kernels (per-field independent, like them)."""
    import torch

    def run(cfg, x):
        y = op(cfg, x.numpy())
        return torch.from_numpy(np.asfortranarray(y))
    return run


def _sharded_main(rank, world, port, nf, out_dir):
    import torch
    from shtb200.distributed import sharded

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = so.create_gauss_config(15, 16)
        a = torch.from_numpy(np.asfortranarray(rand_alm(15, 15, nf, seed=23)))
        f = sharded(_oracle_batch(so.synthesis_batch), cfg, a)                # complex in, real out
        b = sharded(_oracle_batch(so.analysis_batch), cfg, f)                 # real in, complex out
        mine = sharded(_oracle_batch(so.synthesis_batch), cfg, a, gather=False)
        np.save(os.path.join(out_dir, f"f{rank}.npy"), f.numpy())
        np.save(os.path.join(out_dir, f"b{rank}.npy"), b.numpy())
        np.save(os.path.join(out_dir, f"mine{rank}.npy"), mine.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nf", [(2, 5), (2, 1), (3, 7)])
def test_sharded_batch_gathers_whole_result(tmp_path, world, nf):
    """synthesis/analysis_batch_sharded's host logic: each rank transforms its field shard, and
    the all-gather (padded to the largest shard) gives every rank the whole batch, equal to the
    single-process result; without gather each rank keeps its own shard."""
    mp.start_processes(_sharded_main, args=(world, _free_port(), nf, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    cfg = so.create_gauss_config(15, 16)
    a = rand_alm(15, 15, nf, seed=23)
    fref = so.synthesis_batch(cfg, a)
    bref = so.analysis_batch(cfg, fref)
    for r in range(world):
        f = np.load(tmp_path / f"f{r}.npy")
        b = np.load(tmp_path / f"b{r}.npy")
        assert f.shape == fref.shape and np.array_equal(f, fref)
        # the oracle's batched analysis sums over latitudes as a matrix product whose summation
        # order depends on the batch width, so shards agree with the whole batch to rounding
        assert b.shape == bref.shape and np.allclose(b, bref, rtol=0, atol=1e-13 * np.abs(bref).max())
        s0, s1 = shard_range(nf, r, world)
        assert np.array_equal(np.load(tmp_path / f"mine{r}.npy"), fref[:, :, s0:s1])
