"""CPU: the C-ABI library loads, exports every symbol include/shtb200.h declares, and
validates arguments before touching the GPU (no compute calls)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import shtb200 as sht
from shtb200 import _lib
from oracle import sht_oracle as so

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    hdr = (ROOT / "include" / "shtb200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\*?\s+\*?(shtb_[a-z_0-9]+)\s*\(", hdr, re.M)))


def test_header_symbols_exported():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(_lib.SIGNATURES), set(syms) - set(_lib.SIGNATURES)


def test_version_and_gauss_nodes():
    lib = _lib.load()
    assert lib.shtb_version() >= 100
    for n in (1, 2, 7, 64, 513):
        x, w = sht.gauss_nodes(n)
        xo, wo = so.gauss_legendre(n)
        assert np.array_equal(x, xo[::-1]) and np.array_equal(w, wo[::-1])
    assert lib.shtb_gauss_nodes(0, None, None) == _lib.SHTB_ERR_BAD_ARG


@pytest.mark.parametrize("args,msg", [
    ((4, 5, 1, 5, 10), "mmax must be <= lmax"),
    ((4, 4, 1, 4, 10), "nlat >= lmax+1"),
    ((4, 4, 1, 5, 8), "nlon must be >= 2*mmax+1"),
    ((4, 4, 0, 5, 10), "mres must be >= 1"),
    ((-1, 0, 1, 5, 10), "lmax must be >= 0"),
])
def test_plan_validation_errors(args, msg):
    lib = _lib.load()
    lmax, mmax, mres, nlat, nlon = args
    x, w = sht.gauss_nodes(max(nlat, 1))
    h = ctypes.c_void_p()
    rc = lib.shtb_plan_create(ctypes.byref(h), lmax, mmax, mres, nlat, nlon, x.ctypes.data, w.ctypes.data, None,
                              float(nlon), 2 * np.pi / nlon, 0)
    assert rc == _lib.SHTB_ERR_BAD_ARG
    assert msg in lib.shtb_last_error().decode()


def test_null_plan_rejected():
    lib = _lib.load()
    rc = lib.shtb_synthesis(None, None, None, 1, -1, 0, 0, None, 0, None)
    assert rc == _lib.SHTB_ERR_BAD_ARG
    assert lib.shtb_workspace_bytes(None, 0, 1, 0, 0) == 0
    assert lib.shtb_plan_status(None) == _lib.SHTB_ERR_BAD_ARG


def test_newer_entry_points_reject_null_plan():
    """Packed-LM transforms, fused div/vort transforms and the spectral operator validate
    their plan before anything else (no GPU needed)."""
    lib = _lib.load()
    for fn in (lib.shtb_synthesis_packed, lib.shtb_analysis_packed):
        assert fn(None, None, None, 1, -1, _lib.SHTB_F32, _lib.SHTB_PREC_MIXED, None, 0, None) == _lib.SHTB_ERR_BAD_ARG
        assert "plan is NULL" in lib.shtb_last_error().decode()
    for fn in (lib.shtb_synthesis_divvort, lib.shtb_analysis_divvort):
        assert fn(None, None, None, None, None, 1, -1, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, None, 0,
                  None) == _lib.SHTB_ERR_BAD_ARG
        assert "plan is NULL" in lib.shtb_last_error().decode()
    assert lib.shtb_spectral_op(None, _lib.SHTB_SPEC_NEG_LL, None, None, 1, _lib.SHTB_F64,
                                None) == _lib.SHTB_ERR_BAD_ARG
    assert "plan is NULL" in lib.shtb_last_error().decode()


def test_group_arguments_rejected_before_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.shtb_group_create(ctypes.byref(h), None, 0, None) == _lib.SHTB_ERR_BAD_ARG
    assert "n >= 1" in lib.shtb_last_error().decode()
    assert lib.shtb_group_destroy(None) == _lib.SHTB_OK
    assert lib.shtb_group_roundtrip(None, None) == _lib.SHTB_ERR_BAD_ARG
    assert lib.shtb_group_bind(None, None, None, None) == _lib.SHTB_ERR_BAD_ARG
    assert lib.shtb_group_latency_ns(None, None) == _lib.SHTB_ERR_BAD_ARG


def test_group_smooth_nlon_matches_oracle():
    from shtb200.group import smooth_nlon
    for lmax in (31, 63, 100, 255, 300, 511):
        n = smooth_nlon(lmax)
        assert n >= 2 * (lmax + 1) and n == so.smooth_nlon(lmax)
