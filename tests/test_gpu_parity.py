"""GPU parity: the CUDA library (through the C ABI, via the host mirror) against the
SHTns 3.7 golden vectors and the FP64 oracle.

Tolerances: fixtures use their own atol/rtol (3e-12..8e-12, FP32 fixtures 8e-5),
oracle comparisons use relative L2 <= 1e-12 for the FP64 path.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from oracle import sht_oracle as so

from _util import golden, isapprox, rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def both(lmax, nlat, **kw):
    return sht.create_gauss_config(lmax, nlat, **kw), so.create_gauss_config(lmax, nlat, **kw)


def dev(a):
    return sht.to_device(a, torch.complex128 if np.iscomplexobj(a) else torch.float64, 0)


def host(t):
    torch.cuda.synchronize()
    return sht.to_host(t)


# ---------------------------------------------------------------- fixtures
FIXTURES = ["scalar_real_full_gauss_f64", "scalar_batch", "analysis_scalar_full", "sphtor_full_f32",
            "sphtor_batch", "analysis_sphtor_full", "qst_full", "analysis_qst_full"]


@pytest.mark.parametrize("fid", FIXTURES)
def test_shtns37_fixture(fid):
    z, meta = golden()
    m = meta[fid]
    cfg = sht.create_gauss_config(m["lmax"], m["nlat"], mmax=m["mmax"], mres=m["mres"], nlon=m["nphi"],
                                  norm=m["norm"], cs_phase=m["cs_phase"], real_norm=m["real_norm"])
    g = lambda n: z[f"{fid}/{n}"]
    atol, rtol = m["atol"], m["rtol"]
    analysis_only = m["direction"] == "analysis"
    cap = m["capability"]
    if cap in ("scalar_real_full", "scalar_batch"):
        q, v = g("coefficients"), g("field")
        if v.ndim == 2:
            if not analysis_only:
                assert isapprox(host(sht.synthesis(cfg, q)), v, atol, rtol)
            assert isapprox(host(sht.analysis(cfg, v)), q, atol, rtol)
        else:
            if not analysis_only:
                assert isapprox(host(sht.synthesis_batch(cfg, q)), v, atol, rtol)
            assert isapprox(host(sht.analysis_batch(cfg, v)), q, atol, rtol)
    elif cap in ("sphtor_full", "sphtor_batch"):
        S, T, Vt, Vp = g("S"), g("T"), g("Vt"), g("Vp")
        b = S.ndim == 3
        if not analysis_only:
            vt, vp = (sht.synthesis_sphtor_batch if b else sht.synthesis_sphtor)(cfg, S, T)
            assert isapprox(host(vt), Vt, atol, rtol) and isapprox(host(vp), Vp, atol, rtol)
        s, t = (sht.analysis_sphtor_batch if b else sht.analysis_sphtor)(cfg, Vt, Vp)
        assert isapprox(host(s), S, atol, rtol) and isapprox(host(t), T, atol, rtol)
    elif cap == "qst_full":
        Q, S, T, Vr, Vt, Vp = (g(n) for n in "Q S T Vr Vt Vp".split())
        b = Q.ndim == 3
        if not analysis_only:
            vr, vt, vp = (sht.synthesis_qst_batch if b else sht.synthesis_qst)(cfg, Q, S, T)
            assert isapprox(host(vr), Vr, atol, rtol)
            assert isapprox(host(vt), Vt, atol, rtol) and isapprox(host(vp), Vp, atol, rtol)
        q, s, t = (sht.analysis_qst_batch if b else sht.analysis_qst)(cfg, Vr, Vt, Vp)
        assert isapprox(host(q), Q, atol, rtol)
        assert isapprox(host(s), S, atol, rtol) and isapprox(host(t), T, atol, rtol)
    else:
        pytest.fail(cap)


# ---------------------------------------------------------------- oracle sweeps
CASES = [
    dict(lmax=7, nlat=8, nlon=16),
    dict(lmax=7, nlat=9, nlon=15),                 # odd nlat (equator row) and odd nlon
    dict(lmax=12, nlat=14, nlon=27, mmax=9),       # mmax < lmax, nlon with factor 3^3
    dict(lmax=20, nlat=22, nlon=42, mres=2, mmax=20),
    dict(lmax=31, nlat=32, nlon=64),
    dict(lmax=33, nlat=40, nlon=70),               # factor 7
    dict(lmax=47, nlat=48, nlon=202),              # prime factor 101: direct DFT
    dict(lmax=63, nlat=64, nlon=128),
    dict(lmax=100, nlat=101, nlon=216),
    dict(lmax=16, nlat=18, nlon=34, norm="schmidt", cs_phase=False),
    dict(lmax=16, nlat=18, nlon=34, norm="fourpi", real_norm=True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("nf", [1, 3])
def test_scalar_vs_oracle(case, nf):
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg, ocfg = both(lmax, nlat, **c)
    a = rand_alm(lmax, cfg.mmax, nf, seed=1, mres=cfg.mres)
    f_ref = so.synthesis_batch(ocfg, a)
    f = host(sht.synthesis_batch(cfg, a))
    assert rel_l2(f, f_ref) <= TOL64
    g = np.random.default_rng(2).standard_normal((nlat, cfg.nlon, nf))
    assert rel_l2(host(sht.analysis_batch(cfg, g)), so.analysis_batch(ocfg, g)) <= TOL64


@pytest.mark.parametrize("case", CASES[:9], ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("robert", [False, True])
def test_sphtor_vs_oracle(case, robert):
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg, ocfg = both(lmax, nlat, robert_form=robert, **c)
    S = rand_alm(lmax, cfg.mmax, seed=3, power=1.5, mres=cfg.mres, lmin=1)
    T = rand_alm(lmax, cfg.mmax, seed=4, power=1.5, mres=cfg.mres, lmin=1)
    vt_ref, vp_ref = so.synthesis_sphtor(ocfg, S, T)
    vt, vp = sht.synthesis_sphtor(cfg, S, T)
    assert rel_l2(host(vt), vt_ref) <= TOL64 and rel_l2(host(vp), vp_ref) <= TOL64
    rng = np.random.default_rng(5)
    Vt, Vp = rng.standard_normal((nlat, cfg.nlon)), rng.standard_normal((nlat, cfg.nlon))
    s_ref, t_ref = so.analysis_sphtor(ocfg, Vt, Vp)
    s, t = sht.analysis_sphtor(cfg, Vt, Vp)
    assert rel_l2(host(s), s_ref) <= TOL64 and rel_l2(host(t), t_ref) <= TOL64


@pytest.mark.parametrize("ltr", [0, 5, 17])
def test_lcap_truncation(ltr):
    cfg, ocfg = both(24, 26, nlon=50)
    a = rand_alm(24, 24, seed=6)
    assert rel_l2(host(sht.synthesis(cfg, a, lcap=ltr)), so.synthesis(ocfg, a, ltr=ltr)) <= TOL64
    g = np.random.default_rng(7).standard_normal((26, 50))
    assert rel_l2(host(sht.analysis(cfg, g, lcap=ltr)), so.analysis(ocfg, g, ltr=ltr)) <= TOL64
    S, T = rand_alm(24, 24, seed=8, lmin=1), rand_alm(24, 24, seed=9, lmin=1)
    vt, vp = sht.synthesis_sphtor(cfg, S, T, lcap=ltr)
    rt, rp = so.synthesis_sphtor(ocfg, S, T, ltr=ltr)
    if ltr > 0:
        assert rel_l2(host(vt), rt) <= TOL64 and rel_l2(host(vp), rp) <= TOL64
    s, t = sht.analysis_sphtor(cfg, g, g[::-1].copy(), lcap=ltr)
    rs, rt2 = so.analysis_sphtor(ocfg, g, g[::-1].copy(), ltr=ltr)
    if ltr > 0:
        assert rel_l2(host(s), rs) <= TOL64 and rel_l2(host(t), rt2) <= TOL64


@pytest.mark.parametrize("case", [dict(lmax=31, nlat=32, nlon=64), dict(lmax=20, nlat=23, nlon=45, mmax=15)],
                         ids=["l31", "l20-odd"])
def test_phi_scale_quad_vs_oracle(case, monkeypatch):
    """SHTNSKIT_PHI_SCALE=quad (src/SHTnsKit.jl:128-177): synthesis bins scaled by nlon/(2 pi)
    instead of nlon, analysis by 4 pi^2/nlon instead of 2 pi/nlon (the plan's two scalars);
    scalar, sphtor and mixed paths against the oracle built with phi_scale="quad"."""
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    monkeypatch.setenv("SHTNSKIT_PHI_SCALE", "quad")
    cfg = sht.create_gauss_config(lmax, nlat, **c)
    ocfg = so.create_gauss_config(lmax, nlat, phi_scale="quad", **c)
    assert abs(cfg.phi_inv_scale() - ocfg.phi_inv_scale()) == 0.0
    assert abs(ocfg.phi_inv_scale() - cfg.nlon) > 1.0          # really a non-dft scale
    a = rand_alm(lmax, cfg.mmax, 3, seed=61)
    f_ref = so.synthesis_batch(ocfg, a)
    f = host(sht.synthesis_batch(cfg, a))
    assert rel_l2(f, f_ref) <= TOL64
    g = np.random.default_rng(62).standard_normal((nlat, cfg.nlon, 3))
    assert rel_l2(host(sht.analysis_batch(cfg, g)), so.analysis_batch(ocfg, g)) <= TOL64
    # quad synthesis then quad analysis is still the identity on band-limited input
    assert rel_l2(host(sht.analysis_batch(cfg, f)), a) <= 1e-12
    S = rand_alm(lmax, cfg.mmax, seed=63, power=1.5, lmin=1)
    T = rand_alm(lmax, cfg.mmax, seed=64, power=1.5, lmin=1)
    vt, vp = sht.synthesis_sphtor(cfg, S, T)
    rt, rp = so.synthesis_sphtor(ocfg, S, T)
    assert rel_l2(host(vt), rt) <= TOL64 and rel_l2(host(vp), rp) <= TOL64
    s, t = sht.analysis_sphtor(cfg, rt, rp)
    rs, rtt = so.analysis_sphtor(ocfg, rt, rp)
    assert rel_l2(host(s), rs) <= TOL64 and rel_l2(host(t), rtt) <= TOL64
    a32 = a.astype(np.complex64)
    f32 = host(sht.synthesis_batch(cfg, a32, precision="mixed"))
    assert rel_l2(f32, so.synthesis_batch(ocfg, a32.astype(np.complex128))) <= 1e-6
    b32 = host(sht.analysis_batch(cfg, g.astype(np.float32), precision="mixed"))
    assert rel_l2(b32, so.analysis_batch(ocfg, g.astype(np.float32).astype(np.float64))) <= 1e-6


def test_config2_fp64_parity():
    """lmax=511, 512x1024, 16 scalar fields + one sphtor pair, roundtrip vs the oracle at 1e-12."""
    cfg, ocfg = both(511, 512, nlon=1024)
    a = rand_alm(511, 511, 16, seed=0)
    f = sht.synthesis_batch(cfg, a)
    fh = host(f)
    f_ref = so.synthesis_batch(ocfg, a)
    assert rel_l2(fh, f_ref) <= TOL64
    back = host(sht.analysis_batch(cfg, f))
    assert rel_l2(back, so.analysis_batch(ocfg, f_ref)) <= TOL64
    assert rel_l2(back, a) <= 1e-11
    S = rand_alm(511, 511, seed=10, power=1.5, lmin=1)
    T = rand_alm(511, 511, seed=11, power=1.5, lmin=1)
    vt, vp = sht.synthesis_sphtor(cfg, S, T)
    rt, rp = so.synthesis_sphtor(ocfg, S, T)
    assert rel_l2(host(vt), rt) <= TOL64 and rel_l2(host(vp), rp) <= TOL64
    s, t = sht.analysis_sphtor(cfg, vt, vp)
    rs, rtt = so.analysis_sphtor(ocfg, rt, rp)
    assert rel_l2(host(s), rs) <= TOL64 and rel_l2(host(t), rtt) <= TOL64


def test_high_lmax_roundtrip_and_polar_rows():
    """lmax=1023: roundtrip identity, and selected high orders against the oracle (polar underflow rows)."""
    cfg, ocfg = both(1023, 1024, nlon=2048)
    a = rand_alm(1023, 1023, 2, seed=12)
    f = sht.synthesis_batch(cfg, a)
    back = host(sht.analysis_batch(cfg, f))
    assert rel_l2(back, a) <= 1e-11
    # single high orders through the full pipeline vs the oracle
    for m in (0, 700, 1000, 1023):
        am = np.zeros((1024, 1024), dtype=complex)
        am[m:, m] = a[m:, m, 0]
        ref = so.synthesis(ocfg, am)
        assert rel_l2(host(sht.synthesis(cfg, am)), ref) <= TOL64


def test_in_place_and_errors():
    cfg = sht.create_gauss_config(15, 16, nlon=32)
    a = rand_alm(15, 15, seed=13)
    out = sht.julia_empty((16, 32), torch.float64, "cuda:0")
    sht.synthesis_into(cfg, out, a)
    ref = host(sht.synthesis(cfg, a))
    assert np.array_equal(host(out), ref)
    with pytest.raises(sht.DimensionMismatch):
        sht.synthesis(cfg, np.zeros((15, 16), complex))
    with pytest.raises(sht.ArgumentError):
        sht.analysis(cfg, np.zeros((16, 32)), lcap=16)
    with pytest.raises(sht.ArgumentError):
        sht.analysis(cfg, np.zeros((16, 32)), fft_scratch=np.zeros((16, 32), complex))


@pytest.mark.parametrize("nf", [40, 64, 70])
def test_wide_batches_fp64_and_mixed(nf):
    """Batches past 32 and 64 fields take the widest kernel shapes (128-column FP64
    analysis tiles, N = 128 GEMM tiles, several 64-field blocks)."""
    cfg, ocfg = both(31, 32)
    a = rand_alm(31, 31, nf, seed=51)
    f_ref = so.synthesis_batch(ocfg, a)
    assert rel_l2(host(sht.synthesis_batch(cfg, a)), f_ref) <= TOL64
    g = np.random.default_rng(52).standard_normal((32, cfg.nlon, nf))
    b_ref = so.analysis_batch(ocfg, g)
    assert rel_l2(host(sht.analysis_batch(cfg, g)), b_ref) <= TOL64
    f32 = host(sht.synthesis_batch(cfg, a.astype(np.complex64), precision="mixed"))
    assert rel_l2(f32, so.synthesis_batch(ocfg, a.astype(np.complex64).astype(np.complex128))) <= 1e-6
    b32 = host(sht.analysis_batch(cfg, g.astype(np.float32), precision="mixed"))
    assert rel_l2(b32, so.analysis_batch(ocfg, g.astype(np.float32).astype(np.float64))) <= 1e-6


@pytest.mark.gpu
def test_sharded_wrappers_single_process():
    """synthesis/analysis_batch_sharded with no process group: the whole batch on this GPU,
    bit for bit the plain batched calls, and against the oracle (the multi-rank split and
    all-gather are covered on CPU ranks in test_multirank.py)."""
    from shtb200.distributed import analysis_batch_sharded, synthesis_batch_sharded

    cfg = sht.create_gauss_config(31, 32)
    ocfg = so.create_gauss_config(31, 32)
    a = rand_alm(31, 31, 5, seed=31)
    f = synthesis_batch_sharded(cfg, a)
    assert torch.equal(f, sht.synthesis_batch(cfg, a))
    assert rel_l2(host(f), so.synthesis_batch(ocfg, a)) <= TOL64
    b = analysis_batch_sharded(cfg, f)
    assert torch.equal(b, sht.analysis_batch(cfg, f))
    assert rel_l2(host(b), so.analysis_batch(ocfg, host(f))) <= TOL64
