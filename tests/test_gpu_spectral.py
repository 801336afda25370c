"""GPU: diagonal spectral operators (divergence/vorticity maps, the Laplacian) and the
vector transforms with divergence/vorticity spectra, through the C ABI via the host mirror.

Tolerances: the elementwise operators are compared bit for bit with the oracle (same
IEEE operations); the fused transforms at relative L2 <= 1e-12 against the oracle's
composition of the reference functions (FP64 path)."""
import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import DimensionMismatch
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def host(t):
    torch.cuda.synchronize()
    return sht.to_host(t)


def noisy(lmax, mmax, nf, dtype, seed):
    """Random coefficients in every stored entry, forbidden ones included."""
    rng = np.random.default_rng(seed)
    shape = (lmax + 1, mmax + 1) + (() if nf is None else (nf,))
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("mres,nf", [(1, None), (2, None), (1, 3), (3, 2)])
def test_spectral_ops_bitwise(dtype, mres, nf):
    lmax, mmax = 40, 39
    cfg = sht.create_gauss_config(lmax, 42, mmax=mmax, mres=mres)
    ocfg = so.create_gauss_config(lmax, 42, mmax=mmax, mres=mres)
    a = noisy(lmax, mmax, nf, dtype, seed=11 + mres)
    d = host(sht.divergence_from_spheroidal(cfg, a))
    assert d.dtype == dtype and np.array_equal(d, so.neg_ll(ocfg, a))
    assert np.array_equal(host(sht.vorticity_from_toroidal(cfg, a)), so.neg_ll(ocfg, a))
    s = host(sht.spheroidal_from_divergence(cfg, a))
    assert np.array_equal(s, so.inv_neg_ll(ocfg, a))
    assert np.array_equal(host(sht.toroidal_from_vorticity(cfg, a)), so.inv_neg_ll(ocfg, a))


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_in_place_and_laplacian(dtype):
    cfg = sht.create_gauss_config(20, 22, mres=2)
    ocfg = so.create_gauss_config(20, 22, mres=2)
    a = noisy(20, 20, None, np.complex128 if dtype == torch.complex128 else np.complex64, seed=5)
    t = sht.to_device(a, dtype, 0)
    assert sht.divergence_from_spheroidal_into(cfg, t, t) is t
    assert np.array_equal(host(t), so.neg_ll(ocfg, a))
    back = sht.spheroidal_from_divergence_into(cfg, t, t)
    assert back is t and np.array_equal(host(t), so.inv_neg_ll(ocfg, so.neg_ll(ocfg, a)))
    lap = sht.to_device(a, dtype, 0)
    assert sht.gpu_apply_laplacian(cfg, lap) is lap
    assert np.array_equal(host(lap), so.neg_ll(ocfg, a))
    ramp = np.arange(1, 21 * 21 + 1).reshape(21, 21).T.astype(a.dtype)   # CT.(1:N), column-major
    r = sht.to_device(ramp, dtype, 0)
    sht.gpu_apply_laplacian(cfg, r)
    assert np.array_equal(host(r), so.neg_ll(ocfg, ramp))


def test_spectral_op_rejects_bad_shapes():
    cfg = sht.create_gauss_config(10, 12)
    with pytest.raises(DimensionMismatch):
        sht.divergence_from_spheroidal(cfg, np.zeros((12, 11), np.complex128))
    out = sht.to_device(np.zeros((11, 11), np.complex128), torch.complex128, 0)
    with pytest.raises(DimensionMismatch):
        sht.spheroidal_from_divergence_into(cfg, out[:10], np.zeros((11, 11), np.complex128))


@pytest.mark.parametrize("case", [dict(lmax=31, nlat=32), dict(lmax=47, nlat=50, mres=2, mmax=40),
                                  dict(lmax=24, nlat=26, nlon=50, robert_form=True)],
                         ids=["l31", "l47-mres2", "l24-robert"])
def test_divvort_transforms_vs_oracle(case):
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg = sht.create_gauss_config(lmax, nlat, **c)
    ocfg = so.create_gauss_config(lmax, nlat, **c)
    D = rand_alm(lmax, cfg.mmax, seed=21, mres=cfg.mres, lmin=1)
    Z = rand_alm(lmax, cfg.mmax, seed=22, mres=cfg.mres, lmin=1)
    vt_ref, vp_ref = so.synthesis_sphtor(ocfg, so.inv_neg_ll(ocfg, D), so.inv_neg_ll(ocfg, Z))
    vt, vp = sht.synthesis_divvort(cfg, D, Z)
    assert rel_l2(host(vt), vt_ref) <= TOL64 and rel_l2(host(vp), vp_ref) <= TOL64
    rng = np.random.default_rng(23)
    Vt, Vp = rng.standard_normal((nlat, cfg.nlon)), rng.standard_normal((nlat, cfg.nlon))
    s_ref, t_ref = so.analysis_sphtor(ocfg, Vt, Vp)
    d, z = sht.analysis_divvort(cfg, Vt, Vp)
    assert rel_l2(host(d), so.neg_ll(ocfg, s_ref)) <= TOL64
    assert rel_l2(host(z), so.neg_ll(ocfg, t_ref)) <= TOL64
    d0, z0 = host(d), host(z)
    assert d0[0, 0] == 0 and z0[0, 0] == 0


def test_divvort_batch_roundtrip_and_lcap():
    cfg = sht.create_gauss_config(63, 64)
    ocfg = so.create_gauss_config(63, 64)
    D = rand_alm(63, 63, 3, seed=31, lmin=1)
    Z = rand_alm(63, 63, 3, seed=32, lmin=1)
    vt, vp = sht.synthesis_divvort_batch(cfg, D, Z)
    d, z = sht.analysis_divvort_batch(cfg, vt, vp)
    assert rel_l2(host(d), D) <= TOL64 and rel_l2(host(z), Z) <= TOL64
    ltr = 20
    vt_l, vp_l = sht.synthesis_divvort(cfg, D[:, :, 0], Z[:, :, 0], lcap=ltr)
    vt_ref, _ = so.synthesis_sphtor(ocfg, so.inv_neg_ll(ocfg, D[:, :, 0]), so.inv_neg_ll(ocfg, Z[:, :, 0]), ltr=ltr)
    assert rel_l2(host(vt_l), vt_ref) <= TOL64
