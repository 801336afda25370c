"""CPU: the FP64 oracle against the reference's SHTns 3.7 golden vectors, closed-form
harmonics, adjoint identities and the C port (no GPU needed)."""
import math

import numpy as np
import pytest

from oracle import c_oracle as co
from oracle import sht_oracle as so

from _util import golden, isapprox, rand_alm, rel_l2


def cfg_of(m):
    return so.create_gauss_config(m["lmax"], m["nlat"], mmax=m["mmax"], mres=m["mres"], nlon=m["nphi"],
                                  norm=m["norm"], cs_phase=m["cs_phase"], real_norm=m["real_norm"])


@pytest.mark.parametrize("fid", ["scalar_real_full_gauss_f64", "scalar_batch", "analysis_scalar_full"])
def test_scalar_fixtures(fid):
    z, meta = golden()
    m = meta[fid]
    cfg = cfg_of(m)
    q, v = z[f"{fid}/coefficients"], z[f"{fid}/field"]
    batched = v.ndim == 3
    syn = so.synthesis_batch if batched else so.synthesis
    ana = so.analysis_batch if batched else so.analysis
    if m["direction"] != "analysis":
        assert isapprox(syn(cfg, q), v, m["atol"], m["rtol"])
    assert isapprox(ana(cfg, v), q, m["atol"], m["rtol"])


@pytest.mark.parametrize("fid", ["sphtor_full_f32", "sphtor_batch", "analysis_sphtor_full"])
def test_sphtor_fixtures(fid):
    z, meta = golden()
    m = meta[fid]
    cfg = cfg_of(m)
    S, T, Vt, Vp = (z[f"{fid}/{n}"] for n in ("S", "T", "Vt", "Vp"))
    batched = S.ndim == 3
    syn = so.synthesis_sphtor_batch if batched else so.synthesis_sphtor
    ana = so.analysis_sphtor_batch if batched else so.analysis_sphtor
    if m["direction"] != "analysis":
        vt, vp = syn(cfg, S, T)
        assert isapprox(vt, Vt, m["atol"], m["rtol"]) and isapprox(vp, Vp, m["atol"], m["rtol"])
    s, t = ana(cfg, Vt, Vp)
    assert isapprox(s, S, m["atol"], m["rtol"]) and isapprox(t, T, m["atol"], m["rtol"])


@pytest.mark.parametrize("fid", ["qst_full", "analysis_qst_full"])
def test_qst_fixtures_are_scalar_plus_sphtor(fid):
    z, meta = golden()
    m = meta[fid]
    cfg = cfg_of(m)
    Q, S, T, Vr, Vt, Vp = (z[f"{fid}/{n}"] for n in "Q S T Vr Vt Vp".split())
    if Q.ndim == 3:
        q = so.analysis_batch(cfg, Vr)
        s, t = so.analysis_sphtor_batch(cfg, Vt, Vp)
    else:
        q = so.analysis(cfg, Vr)
        s, t = so.analysis_sphtor(cfg, Vt, Vp)
    for got, want in ((q, Q), (s, S), (t, T)):
        assert isapprox(got, want, m["atol"], m["rtol"])


def test_closed_form_low_degree():
    """Y_1^0, Y_1^1 and Y_2^0 in the orthonormal + Condon-Shortley convention."""
    cfg = so.create_gauss_config(4, 6, nlon=10)
    x = cfg.x[:, None]
    phi = 2 * np.pi * np.arange(10)[None, :] / 10
    s = np.sqrt(1 - x ** 2)
    cases = [
        ((1, 0), 1.0, math.sqrt(3 / (4 * math.pi)) * x * np.ones_like(phi)),
        ((2, 0), 1.0, math.sqrt(5 / (16 * math.pi)) * (3 * x ** 2 - 1) * np.ones_like(phi)),
        # real field from a_11 = 1: 2 Re(Y_1^1) with Y_1^1 = -sqrt(3/8pi) sin e^{i phi}
        ((1, 1), 1.0, 2 * (-math.sqrt(3 / (8 * math.pi))) * s * np.cos(phi)),
    ]
    for (l, m_), val, f_exact in cases:
        a = np.zeros((5, 5), complex)
        a[l, m_] = val
        assert np.abs(so.synthesis(cfg, a) - f_exact).max() < 1e-14
        back = so.analysis(cfg, f_exact)
        assert np.abs(back - a).max() < 1e-14


def test_parseval_single_mode():
    cfg = so.create_gauss_config(10, 12, nlon=22)
    for l, m in ((3, 0), (5, 2), (10, 10)):
        a = np.zeros((11, 11), complex)
        a[l, m] = 1.0
        f = so.synthesis(cfg, a)
        energy = np.sum(cfg.w[:, None] * f ** 2) * (2 * np.pi / cfg.nlon)
        assert abs(energy - (1.0 if m == 0 else 2.0)) < 1e-12


def test_high_lmax_row_against_long_double_reference():
    """P_l^m at lmax 2048 for m = 1500 (scaled seed path) against an extended-precision product."""
    x = np.array([0.3, 0.9, 0.999])
    lmax, m = 2048, 1500
    P = so.plm_rows(x, lmax, m)
    # independent: log-space seed then recurrence in numpy longdouble
    ld = np.longdouble
    for i, xi in enumerate(x):
        s = np.sqrt((ld(1) - ld(xi)) * (ld(1) + ld(xi)))
        logp = np.log(ld(so.INV_SQRT_4PI)) + sum(np.log(np.sqrt(ld(2 * j + 1) / ld(2 * j)) * s) for j in range(1, m + 1))
        p2 = ((-1) ** m) * np.exp(logp)
        p1 = np.sqrt(ld(2 * m + 3)) * ld(xi) * p2
        vals = {m: p2, m + 1: p1}
        for l in range(m + 2, lmax + 1):
            a = np.sqrt(ld((2 * l - 1) * (2 * l + 1)) / ld((l - m) * (l + m)))
            b = np.sqrt(ld((2 * l + 1) * (l - 1 - m) * (l - 1 + m)) / ld((2 * l - 3) * (l - m) * (l + m)))
            vals[l] = a * ld(xi) * vals[l - 1] - b * vals[l - 2]
        ref = np.array([float(vals[l]) for l in range(m, lmax + 1)])
        got = P[i, m:]
        big = np.abs(ref) > 1e-250
        assert np.allclose(got[big], ref[big], rtol=2e-11, atol=0)


def _fd_check(fun, grad, x0, h, rng, n=12, rtol=5e-4):
    for _ in range(n):
        d = np.zeros_like(x0)
        idx = tuple(rng.integers(0, s) for s in x0.shape)
        d[idx] = 1.0 if not np.iscomplexobj(x0) or rng.random() < 0.5 else 1j
        fd = (fun(x0 + h * d) - fun(x0 - h * d)) / (2 * h)
        an = np.real(np.sum(np.conj(grad) * d))
        assert abs(fd - an) <= rtol * max(1.0, abs(an)), (fd, an)


@pytest.mark.parametrize("robert", [False, True])
def test_adjoints_against_finite_differences(robert):
    """Zygote-convention gradients g = dL/dRe + i dL/dIm (src/core_transforms.jl:477-652)."""
    rng = np.random.default_rng(0)
    cfg = so.create_gauss_config(9, 11, nlon=20, robert_form=robert)
    a = rand_alm(9, 9, seed=1)
    g = rng.standard_normal((11, 20))
    L = lambda aa: float(np.sum((so.synthesis(cfg, aa) - g) ** 2))
    grad = so.adjoint_synthesis(cfg, 2 * (so.synthesis(cfg, a) - g))
    _fd_check(L, grad, a, 1e-6, rng)
    f = rng.standard_normal((11, 20))
    w = rand_alm(9, 9, seed=2)
    L2 = lambda ff: float(np.real(np.sum(np.conj(w) * so.analysis(cfg, ff))))
    grad2 = np.real(so.adjoint_analysis(cfg, w))
    _fd_check(L2, grad2, f, 1e-6, rng)
    S, T = rand_alm(9, 9, seed=3, lmin=1), rand_alm(9, 9, seed=4, lmin=1)
    gt, gp = rng.standard_normal((11, 20)), rng.standard_normal((11, 20))

    def Lv(SS, TT):
        vt, vp = so.synthesis_sphtor(cfg, SS, TT)
        return float(np.sum((vt - gt) ** 2) + np.sum((vp - gp) ** 2))

    vt, vp = so.synthesis_sphtor(cfg, S, T)
    gS, gT = so.adjoint_synthesis_sphtor(cfg, 2 * (vt - gt), 2 * (vp - gp))
    _fd_check(lambda SS: Lv(SS, T), gS, S, 1e-6, rng)
    _fd_check(lambda TT: Lv(S, TT), gT, T, 1e-6, rng)


def test_c_port_matches_numpy_oracle():
    for (L, nlat, nlon) in [(7, 8, 16), (20, 22, 45), (33, 34, 70), (40, 41, 86)]:
        cfg = so.create_gauss_config(L, nlat, nlon=nlon)
        a = rand_alm(L, L, 2, seed=5)
        assert rel_l2(co.synthesis_batch(cfg, a), so.synthesis_batch(cfg, a)) < 1e-13
        f = np.random.default_rng(6).standard_normal((nlat, nlon, 2))
        assert rel_l2(co.analysis_batch(cfg, f), so.analysis_batch(cfg, f)) < 1e-13
