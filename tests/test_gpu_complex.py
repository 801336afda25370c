"""GPU: complex grids on the FP64 path against the oracle.

`synthesis(cfg, alm; real_output=false)` keeps the bins m >= 0 only (no Hermitian fill)
and returns the complex inverse FFT (src/core_transforms.jl:293-344); `analysis` of a
complex-valued field reads the bins m >= 0 of its FFT (src/core_transforms.jl:169-207).
Both run through `shtb_synthesis_cplx` / `shtb_analysis_cplx`. Bar: relative L2 <= 1e-12.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12

CASES = [
    dict(lmax=15, nlat=16, nlon=32),
    dict(lmax=7, nlat=9, nlon=15),                 # odd nlat (equator row) and odd nlon
    dict(lmax=20, nlat=22, nlon=42, mres=2, mmax=20),
    dict(lmax=33, nlat=40, nlon=70),               # factor 7
    dict(lmax=47, nlat=48, nlon=202),              # prime factor 101: direct DFT
    dict(lmax=16, nlat=18, nlon=34, norm="schmidt", cs_phase=False),
    dict(lmax=255, nlat=256, nlon=512),
]


def host(t):
    torch.cuda.synchronize()
    return sht.to_host(t)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_complex_grids_vs_oracle(case):
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg = sht.create_gauss_config(lmax, nlat, **c)
    ocfg = so.create_gauss_config(lmax, nlat, **c)
    a = rand_alm(lmax, cfg.mmax, seed=81, mres=cfg.mres)
    g = host(sht.synthesis(cfg, a, real_output=False))
    assert np.iscomplexobj(g)
    g_ref = so.synthesis(ocfg, a, real_output=False)
    assert rel_l2(g, g_ref) <= TOL64
    rng = np.random.default_rng(82)
    z = rng.standard_normal((nlat, cfg.nlon)) + 1j * rng.standard_normal((nlat, cfg.nlon))
    assert rel_l2(host(sht.analysis(cfg, z)), so.analysis(ocfg, z)) <= TOL64
    # the complex pair is an identity on coefficients, as in the reference
    assert rel_l2(host(sht.analysis(cfg, g)), so.analysis(ocfg, g_ref)) <= TOL64


@pytest.mark.parametrize("nf", [3, 40])
def test_complex_grids_batched_and_truncated(nf):
    cfg = sht.create_gauss_config(31, 32)
    ocfg = so.create_gauss_config(31, 32)
    a = rand_alm(31, 31, nf, seed=83)
    g = host(sht.synthesis_batch(cfg, a, real_output=False))
    g_ref = np.stack([so.synthesis(ocfg, a[:, :, k], real_output=False) for k in range(nf)], axis=2)
    assert rel_l2(g, g_ref) <= TOL64
    b = host(sht.analysis_batch(cfg, g_ref))
    assert rel_l2(b, np.stack([so.analysis(ocfg, g_ref[:, :, k]) for k in range(nf)], axis=2)) <= TOL64
    for ltr in (0, 9):
        gl = host(sht.synthesis(cfg, a[:, :, 0], real_output=False, lcap=ltr))
        assert rel_l2(gl, so.synthesis(ocfg, a[:, :, 0], real_output=False, ltr=ltr)) <= TOL64
        bl = host(sht.analysis(cfg, g_ref[:, :, 1], lcap=ltr))
        assert rel_l2(bl, so.analysis(ocfg, g_ref[:, :, 1], ltr=ltr)) <= TOL64


def test_complex_grids_reject_mixed_precision():
    cfg = sht.create_gauss_config(7, 8)
    with pytest.raises(sht.BackendUnavailableError):
        sht.synthesis(cfg, rand_alm(7, 7, seed=1).astype(np.complex64), real_output=False, precision="mixed")
    with pytest.raises(sht.BackendUnavailableError):
        sht.analysis(cfg, np.zeros((8, 16), np.complex64), precision="mixed")
