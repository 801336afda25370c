"""GPU: a bounded device wait that runs out.

The tensor-core (mixed-precision) kernels wait on shared-memory barriers with a time
limit. Through the test hook ``shtb_plan_debug_waits`` the host shortens that limit to
1 ms and makes the first CTA's loader leave one chunk's copies unissued, so the wait for
that chunk cannot complete: nothing faults or hangs. The kernel must record the timeout
(``shtb_plan_status`` -> SHTB_ERR_TIMEOUT), drain its own copies and MMAs in flight, free
its tensor memory and return; the next ordinary call on the same plan must then run (its
TMEM allocation succeeds) and be correct against the FP64 oracle.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import _lib
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOLMX = 1e-6


def _status(plan):
    torch.cuda.synchronize()
    with torch.cuda.device(plan.device_index):
        return _lib.load().shtb_plan_status(plan.handle)


# (lmax, nfields, chunk to skip): one chunk per tile on the small case; several chunks per
# tile with copies of later chunks in flight at the abort on the larger one
CASES = [(63, 3, 0), (511, 64, 3)]


@pytest.mark.parametrize("lmax,nf,skip", CASES, ids=["l63-nf3", "l511-nf64"])
def test_wait_timeout_is_reported_and_plan_recovers(lmax, nf, skip):
    lib = _lib.load()
    nlat, nlon = lmax + 1, 2 * (lmax + 1)
    cfg = sht.create_gauss_config(lmax, nlat, nlon=nlon)
    ocfg = so.create_gauss_config(lmax, nlat, nlon=nlon)
    plan = cfg.plan(0)
    a = rand_alm(lmax, lmax, nf, seed=71).astype(np.complex64)
    g = np.random.default_rng(72).standard_normal((nlat, nlon, nf)).astype(np.float32)
    assert _status(plan) == _lib.SHTB_OK
    try:
        _lib.check(lib.shtb_plan_debug_waits(plan.handle, 1_000_000, skip), "debug_waits")
        sht.synthesis_batch(cfg, a, precision="mixed")
        assert _status(plan) == _lib.SHTB_ERR_TIMEOUT, "synthesis: the skipped chunk's wait must run out"
        assert "time limit" in lib.shtb_last_error().decode()
        assert _status(plan) == _lib.SHTB_OK, "the status word is cleared once read"
        sht.analysis_batch(cfg, g, precision="mixed")
        assert _status(plan) == _lib.SHTB_ERR_TIMEOUT, "analysis: the skipped chunk's wait must run out"
    finally:
        _lib.check(lib.shtb_plan_debug_waits(plan.handle, 0, -1), "debug_waits reset")
    # the same plan, ordinary calls: the GEMM kernels allocate TMEM again and are correct
    f = sht.synthesis_batch(cfg, a, precision="mixed")
    b = sht.analysis_batch(cfg, g, precision="mixed")
    torch.cuda.synchronize()
    assert _status(plan) == _lib.SHTB_OK
    pick = [0, nf - 1]
    f_ref = so.synthesis_batch(ocfg, a[:, :, pick].astype(np.complex128))
    assert rel_l2(sht.to_host(f)[:, :, pick], f_ref) <= TOLMX
    b_ref = so.analysis_batch(ocfg, g[:, :, pick].astype(np.float64))
    assert rel_l2(sht.to_host(b)[:, :, pick], b_ref) <= TOLMX


def test_debug_waits_argument_checks():
    lib = _lib.load()
    cfg = sht.create_gauss_config(15, 16)
    plan = cfg.plan(0)
    assert lib.shtb_plan_debug_waits(None, 0, -1) == _lib.SHTB_ERR_BAD_ARG
    assert lib.shtb_plan_debug_waits(plan.handle, 20_000_000_000, -1) == _lib.SHTB_ERR_BAD_ARG
    assert lib.shtb_plan_debug_waits(plan.handle, 0, -1) == _lib.SHTB_OK
