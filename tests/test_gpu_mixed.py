"""GPU parity of the mixed-precision path (tensor-core fp16x3 GEMMs; one- and two-field
syntheses on the FP64 pipes).

Inputs are rounded to FP32 (the path's I/O type); the FP64 oracle runs on the same
rounded inputs. Bar: relative L2 <= 1e-6 against the FP64 result.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOLMX = 1e-6

CASES = [
    dict(lmax=15, nlat=16, nlon=32),
    dict(lmax=31, nlat=33, nlon=64),
    dict(lmax=63, nlat=64, nlon=128),
    dict(lmax=40, nlat=44, nlon=90, mmax=30),
    dict(lmax=30, nlat=32, nlon=64, mres=3, mmax=30),
    dict(lmax=127, nlat=128, nlon=256),
    dict(lmax=20, nlat=22, nlon=42, norm="schmidt", cs_phase=False),
]


def host(t):
    torch.cuda.synchronize()
    return sht.to_host(t)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("nf", [1, 2, 9, 20, 64])
def test_mixed_vs_fp64_oracle(case, nf):
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg = sht.create_gauss_config(lmax, nlat, **c)
    ocfg = so.create_gauss_config(lmax, nlat, **c)
    a = rand_alm(lmax, cfg.mmax, nf, seed=3, mres=cfg.mres).astype(np.complex64).astype(np.complex128)
    f = sht.synthesis_batch(cfg, a.astype(np.complex64), precision="mixed")
    fh = host(f)
    assert fh.dtype == np.float32
    f_ref = so.synthesis_batch(ocfg, a)
    assert rel_l2(fh, f_ref) <= TOLMX
    g = np.random.default_rng(4).standard_normal((nlat, cfg.nlon, nf)).astype(np.float32)
    b = host(sht.analysis_batch(cfg, g, precision="mixed"))
    b_ref = so.analysis_batch(ocfg, g.astype(np.float64))
    assert rel_l2(b, b_ref) <= TOLMX
    cfg.plan(0).status()


@pytest.mark.parametrize("nf", [1, 3])
def test_mixed_lcap(nf):
    cfg = sht.create_gauss_config(40, 42, nlon=81)
    ocfg = so.create_gauss_config(40, 42, nlon=81)
    a = rand_alm(40, 40, nf, seed=5).astype(np.complex64).astype(np.complex128)
    for ltr in (3, 17, 40):
        f = host(sht.synthesis_batch(cfg, a.astype(np.complex64), lcap=ltr, precision="mixed"))
        ref = np.stack([so.synthesis(ocfg, a[:, :, k], ltr=ltr) for k in range(nf)], axis=2)
        assert rel_l2(f, ref) <= TOLMX
        g = np.random.default_rng(6).standard_normal((42, 81, nf)).astype(np.float32)
        b = host(sht.analysis_batch(cfg, g, lcap=ltr, precision="mixed"))
        bref = np.stack([so.analysis(ocfg, g[:, :, k].astype(np.float64), ltr=ltr) for k in range(nf)], axis=2)
        assert rel_l2(b, bref) <= TOLMX


def test_mixed_one_field_high_degree():
    """One field at lmax 511 (FP64-pipe synthesis from the extended-range start records at
    high orders) against the oracle."""
    cfg = sht.create_gauss_config(511, 512, nlon=1024)
    ocfg = so.create_gauss_config(511, 512, nlon=1024)
    a = rand_alm(511, 511, seed=13).astype(np.complex64).astype(np.complex128)
    f = host(sht.synthesis(cfg, a.astype(np.complex64), precision="mixed"))
    assert rel_l2(f, so.synthesis(ocfg, a)) <= TOLMX


def test_mixed_config3_size():
    """lmax=1023, 1024x2048, 64 fields: the mixed roundtrip against the FP64 oracle (the C
    restatement of the reference CPU path) on two of the 64 fields, grid and coefficients,
    and against the FP64 GPU path on all 64, each at <= 1e-6."""
    from oracle import c_oracle as co

    cfg = sht.create_gauss_config(1023, 1024, nlon=2048)
    ocfg = so.create_gauss_config(1023, 1024, nlon=2048)
    a = rand_alm(1023, 1023, 64, seed=7).astype(np.complex64)
    a64 = a.astype(np.complex128)
    f32 = sht.synthesis_batch(cfg, a, precision="mixed")
    f32h = host(f32)
    pick = [0, 37]
    f_ref = co.synthesis_batch(ocfg, a64[:, :, pick])
    for i, k in enumerate(pick):
        assert rel_l2(f32h[:, :, k], f_ref[:, :, i]) <= TOLMX, f"synthesis field {k} vs oracle"
    f64 = sht.synthesis_batch(cfg, a64)
    assert rel_l2(f32h, host(f64)) <= TOLMX
    b32 = sht.analysis_batch(cfg, f32, precision="mixed")
    b32h = host(b32)
    b_ref = co.analysis_batch(ocfg, f32h[:, :, pick].astype(np.float64))
    for i, k in enumerate(pick):
        assert rel_l2(b32h[:, :, k], b_ref[:, :, i]) <= TOLMX, f"analysis field {k} vs oracle"
    b64 = sht.analysis_batch(cfg, f64)
    assert rel_l2(b32h, host(b64)) <= TOLMX
    assert rel_l2(b32h, a64) <= TOLMX
    cfg.plan(0).status()


def test_mixed_field_magnitudes():
    """Fields 50 orders of magnitude apart, an all-zero field, a field whose low degrees
    dominate its high ones by 1e6, and a single nonzero coefficient, in one batch. The f16
    split scales every B row (field, re|im) by its own power of two, so each field meets
    the bar on its own and the zero field stays exactly zero."""
    lmax, nlat, nlon = 63, 64, 128
    cfg = sht.create_gauss_config(lmax, nlat, nlon=nlon)
    ocfg = so.create_gauss_config(lmax, nlat, nlon=nlon)
    nf = 6
    a = rand_alm(lmax, lmax, nf, seed=11)
    a[:, :, 1] *= 1e25
    a[:, :, 2] *= 1e-25
    a[:, :, 3] = 0
    a[:10, :, 4] *= 1e6
    a[:, :, 5] = 0
    a[7, 3, 5] = 2.5 - 1.5j
    a = a.astype(np.complex64).astype(np.complex128)
    f = host(sht.synthesis_batch(cfg, a.astype(np.complex64), precision="mixed"))
    f_ref = so.synthesis_batch(ocfg, a)
    for k in range(nf):
        if k == 3:
            assert not np.any(f[:, :, k]), "zero field"
        else:
            assert rel_l2(f[:, :, k], f_ref[:, :, k]) <= TOLMX, f"synthesis field {k}"
    g = np.random.default_rng(12).standard_normal((nlat, nlon, nf))
    g[:, :, 1] *= 1e25
    g[:, :, 2] *= 1e-25
    g[:, :, 3] = 0
    g[:, :, 4] += 1e6 * np.cos(np.arange(nlon) * 2 * np.pi / nlon)[None, :]
    g[:, :, 5] = 0
    g[5, 9, 5] = 3.0
    g = g.astype(np.float32)
    b = host(sht.analysis_batch(cfg, g, precision="mixed"))
    b_ref = so.analysis_batch(ocfg, g.astype(np.float64))
    for k in range(nf):
        if k == 3:
            assert not np.any(b[:, :, k]), "zero field"
        else:
            assert rel_l2(b[:, :, k], b_ref[:, :, k]) <= TOLMX, f"analysis field {k}"
    cfg.plan(0).status()
