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


# ---------------------------------------------------------------- packed LM layout
PACKED_CASES = [dict(lmax=31, nlat=32), dict(lmax=47, nlat=50, mres=2, mmax=40),
                dict(lmax=20, nlat=22, nlon=45, mmax=12)]


@pytest.mark.parametrize("case", PACKED_CASES, ids=["l31", "l47-mres2", "l20-mmax12"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_packed_equals_dense_bitwise(case, precision):
    """The packed entry points address the coefficients differently but compute the same
    values: bit-identical to pack_lm / unpack_lm around the dense transforms."""
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg = sht.create_gauss_config(lmax, nlat, **c)
    ocfg = so.create_gauss_config(lmax, nlat, **c)
    A = rand_alm(lmax, cfg.mmax, seed=41, mres=cfg.mres)
    if precision == "mixed":
        A = A.astype(np.complex64)
    q = so.pack_lm(ocfg, A)
    f_dense = host(sht.synthesis(cfg, A, precision=precision))
    v = host(sht.synthesis_packed(cfg, q, precision=precision))
    assert np.array_equal(v, f_dense.reshape(-1, order="F"))
    g = np.random.default_rng(42).standard_normal((nlat, cfg.nlon))
    if precision == "mixed":
        g = g.astype(np.float32)
    a_dense = host(sht.analysis(cfg, g, precision=precision))
    qa = host(sht.analysis_packed(cfg, g.reshape(-1, order="F"), precision=precision))
    assert np.array_equal(qa, so.pack_lm(ocfg, a_dense))
    for ltr in (0, lmax // 3):
        vl = host(sht.synthesis_packed_l(cfg, q, ltr, precision=precision))
        assert np.array_equal(vl, host(sht.synthesis(cfg, A, lcap=ltr, precision=precision)).reshape(-1, order="F"))
        ql = host(sht.analysis_packed_l(cfg, g.reshape(-1, order="F"), ltr, precision=precision))
        assert np.array_equal(ql, so.pack_lm(ocfg, host(sht.analysis(cfg, g, lcap=ltr, precision=precision))))


def test_packed_vs_oracle_and_batch():
    cfg = sht.create_gauss_config(40, 42, mres=2)
    ocfg = so.create_gauss_config(40, 42, mres=2)
    A = rand_alm(40, 40, 3, seed=43, mres=2)
    Q = so.pack_lm(ocfg, A)
    V = host(sht.synthesis_packed_batch(cfg, Q))
    assert V.shape == (42 * cfg.nlon, 3)
    for k in range(3):
        assert rel_l2(V[:, k], so.synthesis_packed(ocfg, Q[:, k])) <= TOL64
    back = host(sht.analysis_packed_batch(cfg, V))
    assert rel_l2(back, Q) <= TOL64
    assert np.array_equal(host(sht.pack_lm(cfg, A[:, :, 0])), Q[:, 0])
    assert np.array_equal(host(sht.unpack_lm(cfg, Q[:, 1])), so.unpack_lm(ocfg, Q[:, 1]))
    with pytest.raises(DimensionMismatch):
        sht.synthesis_packed(cfg, Q[:-1, 0])
