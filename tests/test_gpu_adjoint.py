"""GPU adjoints: the four adjoint kernels (through the C ABI) against the oracle's
restatement of the reference rrules, and the differentiation workload (32 fields on
a Gauss grid, lmax=255, nlat=256, nlon=512, FP64) through torch autograd against the
oracle gradient and central finite differences.

Gradient convention (Zygote and PyTorch agree): g = dL/dRe + i dL/dIm for complex
coefficients, g = dL/df for real grids (ext/SHTnsKitAdvancedADExt.jl:55-135,
src/core_transforms.jl:477-652, src/sphtor_transforms.jl:385-452).

Tolerances: kernel-vs-oracle relative L2 <= 1e-12; finite differences (h = 1e-6)
agree to 1e-6 relative to the largest gradient entry checked.
"""
import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import _lib
from shtb200 import transforms as T
from oracle import sht_oracle as so

from _util import rand_alm, rel_l2

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
FD_TOL = 1e-6


def both(lmax, nlat, **kw):
    return sht.create_gauss_config(lmax, nlat, **kw), so.create_gauss_config(lmax, nlat, **kw)


def dev(a):
    return sht.to_device(a, torch.complex128 if np.iscomplexobj(a) else torch.float64, 0)


def host(t):
    torch.cuda.synchronize()
    return sht.to_host(t)


def per_field(fn, *arrays):
    """Apply a single-field oracle function to every trailing-index field."""
    outs = [fn(*(a[:, :, k] for a in arrays)) for k in range(arrays[0].shape[2])]
    if isinstance(outs[0], tuple):
        return tuple(np.stack([o[i] for o in outs], axis=2) for i in range(len(outs[0])))
    return np.stack(outs, axis=2)


ADJ_CASES = [
    dict(lmax=31, nlat=32),
    dict(lmax=20, nlat=24, nlon=45),
    dict(lmax=24, nlat=26, mmax=12, mres=2),
    dict(lmax=15, nlat=16, norm="schmidt"),
    dict(lmax=17, nlat=20, norm="fourpi", cs_phase=False),
]


@pytest.mark.parametrize("case", ADJ_CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_adjoint_kernels_vs_oracle(case):
    c = dict(case)
    lmax, nlat = c.pop("lmax"), c.pop("nlat")
    cfg, ocfg = both(lmax, nlat, **c)
    nf = 3
    rng = np.random.default_rng(11)
    ybar = rng.standard_normal((nlat, cfg.nlon, nf))
    got = host(T.adjoint_synthesis_device(cfg, dev(ybar)))
    assert rel_l2(got, per_field(lambda y: so.adjoint_synthesis(ocfg, y), ybar)) <= TOL64
    abar = rand_alm(lmax, cfg.mmax, nf, seed=12, mres=cfg.mres)
    got = host(T.adjoint_analysis_device(cfg, dev(abar)))
    ref = np.real(per_field(lambda a: so.adjoint_analysis(ocfg, a), abar))
    assert rel_l2(got, ref) <= TOL64


@pytest.mark.parametrize("robert", [False, True])
def test_sphtor_adjoint_kernels_vs_oracle(robert):
    cfg, ocfg = both(23, 24, robert_form=robert)
    nf = 2
    rng = np.random.default_rng(13)
    vtb, vpb = rng.standard_normal((24, cfg.nlon, nf)), rng.standard_normal((24, cfg.nlon, nf))
    S, Tt = T.adjoint_synthesis_sphtor_device(cfg, dev(vtb), dev(vpb))
    S_ref, T_ref = per_field(lambda a, b: so.adjoint_synthesis_sphtor(ocfg, a, b), vtb, vpb)
    assert rel_l2(host(S), S_ref) <= TOL64 and rel_l2(host(Tt), T_ref) <= TOL64
    sb = rand_alm(23, cfg.mmax, nf, seed=14, lmin=1)
    tb = rand_alm(23, cfg.mmax, nf, seed=15, lmin=1)
    vt, vp = T.adjoint_analysis_sphtor_device(cfg, dev(sb), dev(tb))
    vt_ref, vp_ref = per_field(lambda a, b: so.adjoint_analysis_sphtor(ocfg, a, b), sb, tb)
    assert rel_l2(host(vt), np.real(vt_ref)) <= TOL64 and rel_l2(host(vp), np.real(vp_ref)) <= TOL64


def _leaf(a):
    t = dev(a).clone()
    t.requires_grad_(True)
    return t


def _fd_entries(rng, lmax, mmax, nf, n=50, lmin=0):
    """n random (l, m, field, part) entries with l >= max(m, lmin); part 0 = Re, 1 = Im (m > 0)."""
    out = []
    while len(out) < n:
        m = int(rng.integers(0, mmax + 1))
        l = int(rng.integers(max(m, lmin), lmax + 1))
        k = int(rng.integers(0, nf))
        part = 0 if m == 0 else int(rng.integers(0, 2))
        out.append((l, m, k, part))
    return out


def _check_fd(grad, entries, dloss, h=1e-6):
    """Central differences of the loss; dloss(l, m, k, delta) returns L(a+delta) - L(a-delta)."""
    g = np.array([grad[l, m, k].real if p == 0 else grad[l, m, k].imag for l, m, k, p in entries])
    fd = np.array([dloss(l, m, k, h if p == 0 else 1j * h) / (2 * h) for l, m, k, p in entries])
    scale = max(np.abs(g).max(), 1e-300)
    assert np.abs(g - fd).max() <= FD_TOL * scale, (np.abs(g - fd).max(), scale)


def test_differentiation_workload_scalar():
    """Loss sum_k ||synthesis(alm_k) - g_k||^2 on 32 fields; gradient via the adjoint kernel."""
    lmax, nlat, nlon, nf = 255, 256, 512, 32
    cfg, ocfg = both(lmax, nlat, nlon=nlon)
    a = rand_alm(lmax, lmax, nf, seed=0)
    g = np.random.default_rng(1).standard_normal((nlat, nlon, nf))
    at = _leaf(a)
    gt = dev(g)
    launches0 = _lib.load().shtb_launch_count(0)
    f = sht.synthesis_batch(cfg, at)
    loss = ((f - gt) ** 2).sum()
    loss.backward()
    assert _lib.load().shtb_launch_count(0) > launches0
    grad = host(at.grad)
    # oracle gradient: the rrule restated (adjoint synthesis of 2 (f - g)), fields 0..3
    f_h = host(f.detach())
    for k in range(4):
        ref = so.adjoint_synthesis(ocfg, 2 * (f_h[:, :, k] - g[:, :, k]))
        assert rel_l2(grad[:, :, k], ref) <= TOL64
    # central differences of the loss on 50 coefficients; L(a+d) - L(a-d) is formed as
    # sum (f+ - f-) (f+ + f- - 2 g) over the perturbed field to avoid cancellation
    entries = _fd_entries(np.random.default_rng(2), lmax, lmax, nf)

    def dloss(l, m, k, delta):
        ap = a[:, :, k].copy()
        am = a[:, :, k].copy()
        ap[l, m] += delta
        am[l, m] -= delta
        fp = host(sht.synthesis(cfg, ap))
        fm = host(sht.synthesis(cfg, am))
        return float(np.sum((fp - fm) * (fp + fm - 2 * g[:, :, k])))

    _check_fd(grad, entries, dloss)


def test_differentiation_workload_sphtor():
    """Loss ||Vt - gt||^2 + ||Vp - gp||^2 for one spheroidal/toroidal pair (lmax=255)."""
    lmax, nlat, nlon = 255, 256, 512
    cfg, ocfg = both(lmax, nlat, nlon=nlon)
    S = rand_alm(lmax, lmax, seed=3, power=1.5, lmin=1)
    Tt = rand_alm(lmax, lmax, seed=4, power=1.5, lmin=1)
    rng = np.random.default_rng(5)
    gtt, gpp = rng.standard_normal((nlat, nlon)), rng.standard_normal((nlat, nlon))
    s_l, t_l = _leaf(S), _leaf(Tt)
    vt, vp = sht.synthesis_sphtor(cfg, s_l, t_l)
    loss = ((vt - dev(gtt)) ** 2).sum() + ((vp - dev(gpp)) ** 2).sum()
    loss.backward()
    gS, gT = host(s_l.grad), host(t_l.grad)
    vt_h, vp_h = host(vt.detach()), host(vp.detach())
    rS, rT = so.adjoint_synthesis_sphtor(ocfg, 2 * (vt_h - gtt), 2 * (vp_h - gpp))
    assert rel_l2(gS, rS) <= TOL64 and rel_l2(gT, rT) <= TOL64
    ent = _fd_entries(np.random.default_rng(6), lmax, lmax, 1, n=25, lmin=1)

    def make(which):
        def dloss(l, m, k, delta):
            sp, sm, tp, tm = S.copy(), S.copy(), Tt.copy(), Tt.copy()
            if which == "S":
                sp[l, m] += delta
                sm[l, m] -= delta
            else:
                tp[l, m] += delta
                tm[l, m] -= delta
            vtp, vpp = (host(v) for v in sht.synthesis_sphtor(cfg, sp, tp))
            vtm, vpm = (host(v) for v in sht.synthesis_sphtor(cfg, sm, tm))
            return float(np.sum((vtp - vtm) * (vtp + vtm - 2 * gtt)) + np.sum((vpp - vpm) * (vpp + vpm - 2 * gpp)))
        return dloss

    _check_fd(gS[:, :, None], ent, make("S"))
    _check_fd(gT[:, :, None], ent, make("T"))


def test_analysis_gradient_vs_fd():
    """Loss ||analysis(f) - a||^2 w.r.t. the real grid (the rrule's real projection)."""
    lmax, nlat = 31, 32
    cfg, ocfg = both(lmax, nlat)
    rng = np.random.default_rng(8)
    f = rng.standard_normal((nlat, cfg.nlon))
    target = rand_alm(lmax, lmax, seed=9)
    fl = _leaf(f)
    alm = sht.analysis(cfg, fl)
    loss = (torch.abs(alm - dev(target)) ** 2).sum()
    loss.backward()
    grad = host(fl.grad)
    a_h = host(alm.detach())
    ref = np.real(so.adjoint_analysis(ocfg, 2 * (a_h - target)))
    assert rel_l2(grad, ref) <= TOL64
    h = 1e-6
    for _ in range(20):
        i, j = int(rng.integers(0, nlat)), int(rng.integers(0, cfg.nlon))
        fp, fm = f.copy(), f.copy()
        fp[i, j] += h
        fm[i, j] -= h
        ap, am = host(sht.analysis(cfg, fp)), host(sht.analysis(cfg, fm))
        # |ap - t|^2 - |am - t|^2 = Re((ap - am) conj(ap + am - 2 t)), formed without cancellation
        d = float(np.sum(np.real((ap - am) * np.conj(ap + am - 2 * target)))) / (2 * h)
        assert abs(d - grad[i, j]) <= FD_TOL * max(np.abs(grad).max(), 1e-300)


def test_analysis_sphtor_gradient_vs_oracle():
    lmax, nlat = 23, 24
    cfg, ocfg = both(lmax, nlat)
    rng = np.random.default_rng(10)
    Vt, Vp = rng.standard_normal((nlat, cfg.nlon)), rng.standard_normal((nlat, cfg.nlon))
    a, b = _leaf(Vt), _leaf(Vp)
    S, Tt = sht.analysis_sphtor(cfg, a, b)
    loss = (torch.abs(S) ** 2).sum() + 3.0 * (torch.abs(Tt) ** 2).sum()
    loss.backward()
    S_h, T_h = host(S.detach()), host(Tt.detach())
    rvt, rvp = so.adjoint_analysis_sphtor(ocfg, 2 * S_h, 6 * T_h)
    assert rel_l2(host(a.grad), np.real(rvt)) <= TOL64 and rel_l2(host(b.grad), np.real(rvp)) <= TOL64
