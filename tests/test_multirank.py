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
