"""GPU: the allocation-free synthesis entry point against the workspace entry point.

`shtb_synthesis_noalloc` serves hosts that may not allocate device memory while
transforming (their memory belongs to another runtime's pool, or an allocation mid-run
could stall or fail); it keeps its scratch in a library-owned static device array.
This file is collected last so that a failure here leaves every other test already run.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import _lib

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _workspace_synthesis(cfg, plan, a, nf, stream):
    lib = _lib.load()
    f = sht.julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, a.device)
    nb = plan.workspace_bytes(_lib.SHTB_OP_SYNTHESIS, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64)
    ws = torch.empty(nb, dtype=torch.uint8, device=a.device)
    _lib.check(lib.shtb_synthesis(plan.handle, a.data_ptr(), f.data_ptr(), nf, -1, _lib.SHTB_F64,
                                  _lib.SHTB_PREC_FP64, ws.data_ptr(), nb, stream), "synthesis")
    return f


def test_noalloc_synthesis_matches_workspace_entry_point_twice():
    lib = _lib.load()
    torch.cuda.set_device(0)
    cfg = sht.create_gauss_config(63, 64, nlon=128)
    plan = cfg.plan(0)
    stream = torch.cuda.current_stream(0).cuda_stream
    nf = 5
    for call, seed in enumerate((11, 12)):       # two calls in a row, different inputs
        a = sht.to_device(rand_alm(63, 63, nf, seed=seed), torch.complex128, 0)
        ref = _workspace_synthesis(cfg, plan, a, nf, stream)
        out = sht.julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, a.device)
        out.fill_(float("nan"))
        rc = lib.shtb_synthesis_noalloc(plan.handle, a.data_ptr(), out.data_ptr(), nf, -1, stream)
        _lib.check(rc, "synthesis_noalloc")
        torch.cuda.synchronize()
        got, want = sht.to_host(out), sht.to_host(ref)
        assert np.isfinite(got).all(), f"call {call}: unwritten output"
        assert rel_l2(got, want) <= TOL64, f"call {call}"


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
