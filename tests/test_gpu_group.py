"""Uneven batches (``shtb_group_*``): members of different sizes run as persistent grouped
launches (work claimed from device counters) replayed from a CUDA graph must reproduce the
per-member mixed-precision transforms bit for bit, stay within the mixed-precision
tolerance of the FP64 oracle, and keep doing so after autotuning changes the launch shape."""
import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import _lib
from shtb200.group import UnevenBatch, smooth_nlon
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOLMX = 1e-6


def packed_pair_fft(cfg):
    """The library's rule for the packed-pair FP32 FFT kernels (power-of-two nlon in
    64..2048, nlat a multiple of 4); the group runs them in their own persistent kernel."""
    n = cfg.nlon
    return 64 <= n <= 2048 and (n & (n - 1)) == 0 and cfg.nlat % 4 == 0


def fp64_pipe_synthesis(nf):
    """The library's rule for the FP64-pipe Legendre synthesis of the mixed path (one or two
    fields); other members run the packing and the tensor-core synthesis GEMM."""
    return nf <= 2


def members(lmaxes, nfs):
    cfgs = [sht.create_gauss_config(l, l + 1, nlon=smooth_nlon(l)) for l in lmaxes]
    return cfgs, list(nfs)


def fill(batch, seed):
    rng_seeds = iter(range(seed, seed + len(batch.cfgs)))
    host = []
    for c, k, t in zip(batch.cfgs, batch.nf, batch.alm_in):
        a = rand_alm(c.lmax, c.mmax, k, seed=next(rng_seeds)).astype(np.complex64)
        t.copy_(sht.to_device(a, torch.complex64, 0))
        host.append(a)
    return host


def per_member(batch):
    grids, alms = [], []
    for c, a in zip(batch.cfgs, batch.alm_in):
        g = sht.synthesis_batch(c, a, precision="mixed")
        grids.append(g)
        alms.append(sht.analysis_batch(c, g, precision="mixed"))
    torch.cuda.synchronize()
    return grids, alms


def assert_same(batch, grids, alms):
    for t in range(len(batch.cfgs)):
        assert torch.equal(batch.grid[t], grids[t]), f"grid of member {t} differs"
        assert torch.equal(batch.alm_out[t], alms[t]), f"coefficients of member {t} differ"


def test_group_matches_per_member_bitwise():
    lmaxes = [15, 31, 100, 47, 63, 127, 20, 255, 7, 80]
    cfgs, nfs = members(lmaxes, [1, 2, 1, 3, 1, 1, 2, 1, 1, 8])
    b = UnevenBatch(cfgs, nfs)
    host = fill(b, 100)
    launches0 = _lib.load().shtb_launch_count(0)
    b.roundtrip()
    torch.cuda.synchronize()
    # start marker; FP64-pipe synthesis (one- and two-field members); packing and synthesis
    # GEMM (the others); one FFT kernel per direction and FFT kind; analysis GEMM (all)
    kinds = len({packed_pair_fft(c) for c in cfgs})
    synth = {fp64_pipe_synthesis(k) for k in nfs}
    assert kinds == 2 and synth == {True, False}
    assert _lib.load().shtb_launch_count(0) - launches0 == 1 + 1 + 2 + 2 * kinds + 1
    b.status()
    grids, alms = per_member(b)
    assert_same(b, grids, alms)
    # the FP64 oracle, two members: the grouped synthesis, and the grouped analysis of the
    # grid that the group itself produced
    for t in (1, 7):
        oc = so.create_gauss_config(lmaxes[t], lmaxes[t] + 1, nlon=smooth_nlon(lmaxes[t]))
        g = sht.to_host(b.grid[t])
        ref = so.synthesis_batch(oc, host[t].astype(np.complex128))
        assert rel_l2(g, ref) <= TOLMX
        aref = so.analysis_batch(oc, g.astype(np.float64))
        assert rel_l2(sht.to_host(b.alm_out[t]), aref) <= TOLMX
    # replays and direct launches agree
    b.alm_out[0].zero_()
    b.roundtrip()
    b.launch()
    torch.cuda.synchronize()
    assert_same(b, grids, alms)
    lat = b.latencies_ns()
    assert np.all(lat > 0)


def test_group_autotune_keeps_results():
    lmaxes = [63, 31, 127, 15]
    cfgs, nfs = members(lmaxes, [2, 1, 1, 4])
    b = UnevenBatch(cfgs, nfs)
    fill(b, 200)
    h, fft_ctas, gemm_ctas = b.autotune()
    assert h in (4, 8, 16) and fft_ctas >= 1 and gemm_ctas >= 1
    b.roundtrip()
    torch.cuda.synchronize()
    b.status()
    grids, alms = per_member(b)
    assert_same(b, grids, alms)


def test_uneven_workload_sample():
    """32 members drawn like the uneven-batching workload (lmax uniform in 31..511, seed 7)."""
    rng = np.random.default_rng(7)
    lmaxes = [int(v) for v in rng.integers(31, 512, size=32)]
    cfgs, nfs = members(lmaxes, [1] * 32)
    b = UnevenBatch(cfgs, nfs)
    fill(b, 300)
    b.autotune()
    b.roundtrip()
    torch.cuda.synchronize()
    b.status()
    grids, alms = per_member(b)
    assert_same(b, grids, alms)


def test_group_rejects_bad_members():
    cfg = sht.create_gauss_config(31, 32, mres=2, mmax=14)
    with pytest.raises(Exception):
        UnevenBatch([cfg], 1)
    cfg = sht.create_gauss_config(31, 32)
    with pytest.raises(Exception):
        UnevenBatch([cfg], 9)
