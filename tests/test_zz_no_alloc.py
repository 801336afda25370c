"""GPU: the allocation-free synthesis entry point.

`shtb_synthesis_noalloc` serves hosts that may not allocate device memory while
transforming (their memory belongs to another runtime's pool, or an allocation mid-run
could stall or fail); it keeps its scratch in a library-owned static device array whose
address the plan resolved when it was created. Its results are checked against the FP64
oracle and against the workspace entry point, on two calls in a row, and a call after the
first must leave the device's free memory unchanged.
This file is collected last so that a failure here leaves every other test already run.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import _lib
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _workspace_synthesis(cfg, plan, a, nf, ltr, stream):
    lib = _lib.load()
    f = sht.julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, a.device)
    nb = plan.workspace_bytes(_lib.SHTB_OP_SYNTHESIS, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64)
    ws = torch.empty(nb, dtype=torch.uint8, device=a.device)
    _lib.check(lib.shtb_synthesis(plan.handle, a.data_ptr(), f.data_ptr(), nf, ltr, _lib.SHTB_F64,
                                  _lib.SHTB_PREC_FP64, ws.data_ptr(), nb, stream), "synthesis")
    return f


@pytest.mark.parametrize("ltr", [-1, 40])
def test_noalloc_synthesis_matches_oracle_and_workspace_entry_point_twice(ltr):
    lib = _lib.load()
    torch.cuda.set_device(0)
    cfg = sht.create_gauss_config(63, 64, nlon=128)
    ocfg = so.create_gauss_config(63, 64, nlon=128)
    plan = cfg.plan(0)
    stream = torch.cuda.current_stream(0).cuda_stream
    nf = 5
    for call, seed in enumerate((11, 12)):       # two calls in a row, different inputs
        ah = rand_alm(63, 63, nf, seed=seed)
        a = sht.to_device(ah, torch.complex128, 0)
        ref = _workspace_synthesis(cfg, plan, a, nf, ltr, stream)
        out = sht.julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, a.device)
        out.fill_(float("nan"))
        rc = lib.shtb_synthesis_noalloc(plan.handle, a.data_ptr(), out.data_ptr(), nf, ltr, stream)
        _lib.check(rc, "synthesis_noalloc")
        torch.cuda.synchronize()
        got, want = sht.to_host(out), sht.to_host(ref)
        assert np.isfinite(got).all(), f"call {call}: unwritten output"
        cap = 63 if ltr < 0 else ltr
        oracle = np.stack([so.synthesis(ocfg, ah[:, :, k], ltr=cap) for k in range(nf)], axis=2)
        assert rel_l2(got, oracle) <= TOL64, f"call {call} vs oracle"
        assert rel_l2(got, want) <= TOL64, f"call {call} vs workspace entry point"


def test_noalloc_call_takes_no_device_memory():
    lib = _lib.load()
    torch.cuda.set_device(0)
    cfg = sht.create_gauss_config(127, 128, nlon=256)
    plan = cfg.plan(0)
    stream = torch.cuda.current_stream(0).cuda_stream
    nf = 8
    a = sht.to_device(rand_alm(127, 127, nf, seed=21), torch.complex128, 0)
    out = sht.julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, a.device)
    _lib.check(lib.shtb_synthesis_noalloc(plan.handle, a.data_ptr(), out.data_ptr(), nf, -1, stream), "warm-up")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        _lib.check(lib.shtb_synthesis_noalloc(plan.handle, a.data_ptr(), out.data_ptr(), nf, -1, stream), "call")
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_rejects_requests_beyond_its_scratch():
    lib = _lib.load()
    cfg = sht.create_gauss_config(511, 512, nlon=1024)   # 4 MiB of scratch per field
    plan = cfg.plan(0)
    nf = 64
    a = torch.zeros((nf, 512, 512), dtype=torch.complex128, device="cuda:0")
    f = torch.zeros((nf, 1024, 512), dtype=torch.float64, device="cuda:0")
    rc = lib.shtb_synthesis_noalloc(plan.handle, a.data_ptr(), f.data_ptr(), nf, -1,
                                    torch.cuda.current_stream(0).cuda_stream)
    assert rc == _lib.SHTB_ERR_WORKSPACE
    assert "static scratch holds" in lib.shtb_last_error().decode()
