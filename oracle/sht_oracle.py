"""FP64 CPU oracle for the scalar and spheroidal/toroidal spherical harmonic transforms.

TEST INFRASTRUCTURE ONLY. This module restates, in NumPy, the algorithm of
SHTnsKit.jl v3.0.0 for the Gauss-Legendre scalar and sphtor transforms and their
adjoints. Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the checker
or as the timed reference arm. The product path (the CUDA library behind the
C ABI) never calls into this file.

Parity pin: the restatement is checked against the SHTns 3.7 golden vectors that
the reference ships (``test/fixtures/shtns37``), converted by
``tests/golden/make_golden.py`` into ``tests/golden/shtns37_hotpath.npz``, and
against closed-form l<=2 harmonics.

Conventions (reference file:line, paths relative to the SHTnsKit.jl project):
- Gauss nodes/weights: ``src/legendre.jl:956-1003`` (Newton on P_n, tol 1e-15,
  50 iterations), stored north-pole first (``src/config.jl:639``).
- Orthonormal + Condon-Shortley P̄_l^m with the 2^±480 seed exponent:
  ``src/legendre.jl:197-322``.
- dθP̄ and P̄/sinθ rows: ``src/legendre.jl:326-338`` and ``:478-555``.
- Scalar pipeline: ``src/core_transforms.jl:169-344`` with the contractions of
  ``src/kernels.jl:24-65``; φ scales ``src/SHTnsKit.jl:128-177``.
- Vector pipeline: ``src/sphtor_transforms.jl:162-289`` and ``src/kernels.jl:127-215``.
- Adjoints: ``src/core_transforms.jl:477-652`` and ``src/sphtor_transforms.jl:385-452``.
- Normalization boundary: ``src/normalization.jl:142-150`` and ``:313-334``.

Layouts are the reference's column-major ones expressed as NumPy arrays with
C order reversed: a grid is ``f[..., nlat, nlon]`` is NOT used; instead every
array here is indexed exactly like the Julia array, ``f[i, j]`` (latitude i,
longitude j) and ``alm[l, m]``, with an optional trailing field index. Device
buffers use the Fortran-order bytes of these arrays (latitude fastest).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

INV_SQRT_4PI = 0.28209479177387814          # src/legendre.jl:197
POLE_TOLERANCE = 100 * np.finfo(np.float64).eps   # src/legendre.jl:77 × eps
SCALE_BITS = 480                             # src/legendre.jl:207
TINY = math.ldexp(1.0, -SCALE_BITS)
HUGE = math.ldexp(1.0, SCALE_BITS)
SHIFT = 2 * SCALE_BITS


# ---------------------------------------------------------------------------
# Quadrature and configuration
# ---------------------------------------------------------------------------

def gauss_legendre(n: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Legendre nodes/weights, ascending x, as ``src/legendre.jl:956-1003``."""
    if n <= 0:
        raise ValueError("n must be positive")
    x = np.empty(n)
    w = np.empty(n)
    for k in range(1, (n + 1) // 2 + 1):
        z = math.cos(math.pi * (k - 0.25) / (n + 0.5))
        for _ in range(50):
            pnm1, pn = 1.0, z
            for l in range(2, n + 1):
                pnm1, pn = pn, ((2 * l - 1) * z * pn - (l - 1) * pnm1) / l
            pd = n * (z * pn - pnm1) / (z * z - 1.0)
            z1 = z
            z -= pn / pd
            if abs(z - z1) < 1e-15:
                break
        pnm1, pn = 1.0, z
        for l in range(2, n + 1):
            pnm1, pn = pn, ((2 * l - 1) * z * pn - (l - 1) * pnm1) / l
        pd = n * (z * pn - pnm1) / (z * z - 1.0)
        x[k - 1] = -z
        x[n - k] = z
        wk = 2.0 / ((1.0 - z * z) * pd * pd)
        w[k - 1] = wk
        w[n - k] = wk
    return x, w


def norm_scale_from_orthonormal(l: int, m: int, norm: str) -> float:
    """Multiplier to the configured normalization (``src/normalization.jl:100-131``)."""
    if norm == "orthonormal":
        return 1.0
    if norm == "fourpi":
        return math.sqrt(4 * math.pi)
    if norm == "schmidt":
        return math.sqrt(4 * math.pi / (2 * l + 1))
    raise ValueError(f"Unsupported normalization: {norm}")


@dataclass
class Config:
    """Gauss grid configuration mirroring ``create_gauss_config`` (``src/config.jl:633-655``)."""
    lmax: int
    nlat: int
    mmax: int
    mres: int
    nlon: int
    norm: str = "orthonormal"
    cs_phase: bool = True
    real_norm: bool = False
    robert_form: bool = False
    phi_scale: str = "dft"
    x: np.ndarray = field(default=None, repr=False)
    w: np.ndarray = field(default=None, repr=False)

    @property
    def canonical(self) -> bool:
        return self.norm == "orthonormal" and not self.real_norm and self.cs_phase

    def phi_inv_scale(self) -> float:            # src/SHTnsKit.jl:141-159
        return self.nlon / (2 * math.pi) if self.phi_scale == "quad" else float(self.nlon)

    def analysis_phi_scale(self) -> float:       # src/SHTnsKit.jl:177
        return (2 * math.pi / self.nlon) * self.nlon / self.phi_inv_scale()

    def scale_matrix(self) -> np.ndarray:
        """coefficient_scale_to_canonical per (l, m) (``src/normalization.jl:142-147``)."""
        s = np.ones((self.lmax + 1, self.mmax + 1))
        for m in range(self.mmax + 1):
            for l in range(m, self.lmax + 1):
                v = norm_scale_from_orthonormal(l, m, self.norm)
                if self.real_norm and m > 0:
                    v *= 1.0 / math.sqrt(2.0)
                if not self.cs_phase:
                    v *= (-1.0) ** m
                s[l, m] = v
        return s

    def sint(self) -> np.ndarray:
        return np.sqrt(np.maximum(0.0, (1.0 - self.x) * (1.0 + self.x)))


def default_nlon(lmax: int) -> int:
    """Next even integer >= 2*lmax+1 (``_default_nlon``, ``src/config.jl:76-80``)."""
    n = 2 * lmax + 1
    return n + (n & 1)


def smooth_nlon(lmax: int) -> int:
    """Smallest 2^a 3^b 5^c >= 2(lmax+1): the uneven-batch grid rule."""
    n = 2 * (lmax + 1)
    while True:
        k = n
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return n
        n += 1


def create_gauss_config(lmax: int, nlat: int, *, mmax: int | None = None, mres: int = 1,
                        nlon: int | None = None, norm: str = "orthonormal",
                        cs_phase: bool = True, real_norm: bool = False,
                        robert_form: bool = False, phi_scale: str = "dft") -> Config:
    mmax = lmax if mmax is None else mmax
    nlon = default_nlon(lmax) if nlon is None else nlon
    validate_layout(lmax, mmax, mres, nlat, nlon)
    x, w = gauss_legendre(nlat)
    cfg = Config(lmax, nlat, mmax, mres, nlon, norm, cs_phase, real_norm, robert_form, phi_scale)
    cfg.x = x[::-1].copy()      # north-pole first (src/config.jl:639)
    cfg.w = w[::-1].copy()
    return cfg


def validate_layout(lmax, mmax, mres, nlat, nlon):
    """``_validate_spectral_layout`` (``src/config.jl:465-481``) for Gauss grids."""
    if lmax < 0:
        raise ValueError(f"lmax must be ≥ 0, got {lmax}")
    if mmax < 0:
        raise ValueError(f"mmax must be ≥ 0, got {mmax}")
    if mmax > lmax:
        raise ValueError(f"mmax must be ≤ lmax, got mmax={mmax}, lmax={lmax}")
    if mres < 1:
        raise ValueError(f"mres must be ≥ 1, got {mres}")
    if nlat < 1:
        raise ValueError(f"nlat must be ≥ 1, got {nlat}")
    if nlat < lmax + 1:
        raise ValueError(f"Gauss–Legendre quadrature requires nlat ≥ lmax+1, got nlat={nlat} and lmax={lmax}")
    if nlon < 2 * mmax + 1:
        raise ValueError(f"nlon must be ≥ 2*mmax+1 = {2*mmax+1} to resolve every azimuthal order, got nlon={nlon}")


# ---------------------------------------------------------------------------
# Associated Legendre rows (vectorised over an array of x)
# ---------------------------------------------------------------------------

def _rec_coeffs(l: int, m: int) -> tuple[float, float]:
    a = math.sqrt((float(2 * l - 1) * float(2 * l + 1)) / (float(l - m) * float(l + m)))
    b = math.sqrt((float(2 * l + 1) * float(l - 1 - m) * float(l - 1 + m))
                  / (float(2 * l - 3) * float(l - m) * float(l + m)))
    return a, b


def sectoral_seed(s: np.ndarray, m: int) -> tuple[np.ndarray, np.ndarray]:
    """(p, e) with P̄_m^m = p·2^e, blocks of 8 factors (``src/legendre.jl:252-271``)."""
    pmm = np.full(s.shape, INV_SQRT_4PI)
    e = np.zeros(s.shape, dtype=np.int64)
    up = math.ldexp(1.0, SHIFT)
    k = 1
    while k <= m:
        kend = min(k + 7, m)
        for j in range(k, kend + 1):
            pmm = (-math.sqrt(float(2 * j + 1) / float(2 * j)) * s) * pmm
        while True:
            small = (np.abs(pmm) < TINY) & (pmm != 0)
            if not small.any():
                break
            with np.errstate(over="ignore"):
                pmm = np.where(small, pmm * up, pmm)
            e = np.where(small, e - SHIFT, e)
        k = kend + 1
    return pmm, e


def plm_rows(x: np.ndarray, lmax: int, m: int) -> np.ndarray:
    """P̄_l^m(x) for l = 0..lmax (zeros for l<m), rows over x: shape (len(x), lmax+1).

    Restates ``Plm_norm_row!`` including the scaled branch (``src/legendre.jl:233-322``).
    """
    x = np.asarray(x, dtype=np.float64)
    P = np.zeros((x.size, lmax + 1))
    if lmax < m:
        return P
    s = np.sqrt(np.maximum(0.0, (1.0 - x) * (1.0 + x)))
    pmm, e = sectoral_seed(s, m)
    factor = np.ldexp(1.0, e)
    P[:, m] = pmm * factor
    if lmax == m:
        return P
    p2 = pmm.copy()
    p1 = math.sqrt(float(2 * m + 3)) * x * pmm
    P[:, m + 1] = p1 * factor
    scaled = e != 0
    up = math.ldexp(1.0, SHIFT)
    down = math.ldexp(1.0, -SHIFT)
    for l in range(m + 2, lmax + 1):
        a, b = _rec_coeffs(l, m)
        p = a * x * p1 - b * p2
        P[:, l] = p * factor
        p2, p1 = p1, p
        if scaled.any():
            mag = np.maximum(np.abs(p2), np.abs(p1))
            hi = scaled & (mag > HUGE)
            lo = scaled & ~hi & (mag < TINY) & (mag != 0)
            if hi.any():
                p2 = np.where(hi, p2 * down, p2)
                p1 = np.where(hi, p1 * down, p1)
                e = np.where(hi, e + SHIFT, e)
            if lo.any():
                p2 = np.where(lo, p2 * up, p2)
                p1 = np.where(lo, p1 * up, p1)
                e = np.where(lo, e - SHIFT, e)
            scaled = e != 0
            factor = np.ldexp(1.0, e)
    return P


def plm_dtheta_rows(x: np.ndarray, lmax: int, m: int):
    """(P̄, dθP̄, P̄/sinθ) rows, each (len(x), lmax+1) (``src/legendre.jl:478-555``)."""
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    dP = np.zeros((n, lmax + 1))
    Ps = np.zeros((n, lmax + 1))
    s = np.sqrt(np.maximum(0.0, (1.0 - x) * (1.0 + x)))
    interior = (s >= POLE_TOLERANCE) & (lmax >= m)
    if m == 0:
        P = plm_rows(x, lmax, 0)
        d = np.zeros(n)
        for l in range(1, lmax + 1):      # _zonal_dtheta_step (src/legendre.jl:326-338)
            d = math.sqrt(float(2 * l + 1) / float(2 * l - 1)) * (x * d - float(l) * s * P[:, l - 1])
            dP[:, l] = np.where(interior, d, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv_s = np.where(interior, 1.0 / np.where(interior, s, 1.0), 0.0)
        Ps[:, :] = np.where(interior[:, None], P * inv_s[:, None], 0.0)
        return P, dP, Ps
    Pb = plm_rows(x, lmax + 1, m)
    P = Pb[:, : lmax + 1].copy()
    if lmax < m:
        return P, dP, Ps
    with np.errstate(divide="ignore", invalid="ignore"):
        inv_s = np.where(interior, 1.0 / np.where(interior, s, 1.0), 0.0)
    for l in range(m, lmax + 1):
        dl1m = math.sqrt(max(0.0, float((l + 1) ** 2 - m * m) / float(4 * (l + 1) ** 2 - 1)))
        dlm = 0.0 if (l == 0 or l == m) else math.sqrt(max(0.0, float(l * l - m * m) / float(4 * l * l - 1)))
        pm1 = Pb[:, l - 1] if l > 0 else 0.0
        dP[:, l] = (float(l) * dl1m * Pb[:, l + 1] - float(l + 1) * dlm * pm1) * inv_s
        Ps[:, l] = Pb[:, l] * inv_s
    pole = ~interior
    if pole.any():
        dP[pole, :] = 0.0
        Ps[pole, :] = 0.0
        if m == 1:
            for l in range(1, lmax + 1):
                mag = 0.5 * INV_SQRT_4PI * math.sqrt(float(2 * l + 1) * l * (l + 1))
                north = x[pole] > 0
                sdp = -1.0 if (l + 1) % 2 == 1 else 1.0
                sps = -1.0 if l % 2 == 1 else 1.0
                dP[pole, l] = np.where(north, -mag, sdp * mag)
                Ps[pole, l] = np.where(north, -mag, sps * mag)
    return P, dP, Ps


# ---------------------------------------------------------------------------
# Transforms (single field: alm (L+1, M+1) complex; grid (nlat, nlon) real)
# ---------------------------------------------------------------------------

def _mvals(cfg: Config):
    return range(0, cfg.mmax + 1, cfg.mres)


def _to_internal(cfg, alm):
    return alm if cfg.canonical else alm * cfg.scale_matrix()


def _externalize(cfg, alm):
    if cfg.canonical:
        return alm
    out = alm / cfg.scale_matrix()
    for m in range(cfg.mmax + 1):
        out[:m, m] = 0
    return out


def _hermitian_fill(cfg, F):
    for m in range(1, cfg.mmax + 1):
        F[:, cfg.nlon - m] = np.conj(F[:, m])


def synthesis(cfg: Config, alm: np.ndarray, real_output: bool = True, ltr: int | None = None):
    """Scalar synthesis (``src/core_transforms.jl:294-344``; kernel ``src/kernels.jl:57-65``)."""
    ltr = cfg.lmax if ltr is None else min(ltr, cfg.lmax)
    a = _to_internal(cfg, np.asarray(alm, dtype=np.complex128))
    F = np.zeros((cfg.nlat, cfg.nlon), dtype=np.complex128)
    for m in _mvals(cfg):
        if m > ltr or not np.any(a[m:ltr + 1, m]):
            continue
        P = plm_rows(cfg.x, cfg.lmax, m)
        F[:, m] = cfg.phi_inv_scale() * (P[:, m:ltr + 1] @ a[m:ltr + 1, m])
    if real_output:
        _hermitian_fill(cfg, F)
    f = np.fft.ifft(F, axis=1)
    return f.real.copy() if real_output else f


def analysis(cfg: Config, f: np.ndarray, ltr: int | None = None):
    """Scalar analysis (``src/core_transforms.jl:169-207``; kernel ``src/kernels.jl:33-40``)."""
    ltr = cfg.lmax if ltr is None else min(ltr, cfg.lmax)
    F = np.fft.fft(np.asarray(f), axis=1)
    alm = np.zeros((cfg.lmax + 1, cfg.mmax + 1), dtype=np.complex128)
    sc = cfg.analysis_phi_scale()
    for m in _mvals(cfg):
        if m > ltr:
            continue
        P = plm_rows(cfg.x, cfg.lmax, m)
        alm[m:ltr + 1, m] = ((cfg.w * sc)[:, None] * P[:, m:ltr + 1]).T @ F[:, m]
    return _externalize(cfg, alm)


def synthesis_sphtor(cfg: Config, S: np.ndarray, T: np.ndarray, real_output: bool = True,
                     ltr: int | None = None):
    """Vector synthesis (``src/sphtor_transforms.jl:178-241``, ``src/kernels.jl:155-169``)."""
    ltr = cfg.lmax if ltr is None else min(ltr, cfg.lmax)
    S = _to_internal(cfg, np.asarray(S, dtype=np.complex128))
    T = _to_internal(cfg, np.asarray(T, dtype=np.complex128))
    Ft = np.zeros((cfg.nlat, cfg.nlon), dtype=np.complex128)
    Fp = np.zeros_like(Ft)
    inv = cfg.phi_inv_scale()
    for m in _mvals(cfg):
        lo = max(1, m)
        if lo > ltr:
            continue
        _, dP, Ps = plm_dtheta_rows(cfg.x, cfg.lmax, m)
        dY = dP[:, lo:ltr + 1]
        Ys = Ps[:, lo:ltr + 1]
        s = S[lo:ltr + 1, m]
        t = T[lo:ltr + 1, m]
        Ft[:, m] = inv * (dY @ s - 1j * m * (Ys @ t))
        Fp[:, m] = inv * (1j * m * (Ys @ s) + dY @ t)
    if real_output:
        _hermitian_fill(cfg, Ft)
        _hermitian_fill(cfg, Fp)
    vt = np.fft.ifft(Ft, axis=1)
    vp = np.fft.ifft(Fp, axis=1)
    if real_output:
        vt, vp = vt.real.copy(), vp.real.copy()
    if cfg.robert_form:
        st = cfg.sint()[:, None]
        vt = vt * st
        vp = vp * st
    return vt, vp


def analysis_sphtor(cfg: Config, Vt: np.ndarray, Vp: np.ndarray, ltr: int | None = None):
    """Vector analysis (``src/sphtor_transforms.jl:252-289``, ``src/kernels.jl:205-215``)."""
    ltr = cfg.lmax if ltr is None else min(ltr, cfg.lmax)
    Ft = np.fft.fft(np.asarray(Vt), axis=1)
    Fp = np.fft.fft(np.asarray(Vp), axis=1)
    if cfg.robert_form:
        st = cfg.sint()
        inv = np.where(st > 0, 1.0 / np.where(st > 0, st, 1.0), 1.0)[:, None]
        Ft = Ft * inv
        Fp = Fp * inv
    S = np.zeros((cfg.lmax + 1, cfg.mmax + 1), dtype=np.complex128)
    T = np.zeros_like(S)
    sc = cfg.analysis_phi_scale()
    for m in _mvals(cfg):
        lo = max(1, m)
        if lo > ltr:
            continue
        _, dP, Ps = plm_dtheta_rows(cfg.x, cfg.lmax, m)
        ls = np.arange(lo, ltr + 1)
        c = 1.0 / (ls * (ls + 1.0))
        wdY = (cfg.w * sc)[:, None] * dP[:, lo:ltr + 1]
        wYs = (cfg.w * sc)[:, None] * Ps[:, lo:ltr + 1]
        ft = Ft[:, m]
        fp = Fp[:, m]
        # conj(i m Y/s) = -i m Y/s
        S[lo:ltr + 1, m] = c * (wdY.T @ ft - 1j * m * (wYs.T @ fp))
        T[lo:ltr + 1, m] = c * (1j * m * (wYs.T @ ft) + wdY.T @ fp)
    return _externalize(cfg, S), _externalize(cfg, T)


# ---------------------------------------------------------------------------
# Packed LM layout, src/layout.jl:88-101 (nlm_calc), :143-162 (LM_index), :282-339
# (unpack_lm / pack_lm); also decodes the packed golden fixtures. Packed transforms,
# src/transforms.jl:125-155 and :183-227. Trailing axes (fields) pass through.
# ---------------------------------------------------------------------------

def nlm_calc(lmax: int, mmax: int, mres: int) -> int:
    return 0 if mmax > lmax else sum(lmax - m + 1 for m in range(0, mmax + 1, mres))


def lm_index(lmax: int, mres: int, l: int, m: int) -> int:
    im = m // mres
    return ((im * (2 * lmax + 2 - (im + 1) * mres)) >> 1) + l


def pack_lm(cfg: Config, A: np.ndarray) -> np.ndarray:
    A = np.asarray(A)
    q = np.zeros((nlm_calc(cfg.lmax, cfg.mmax, cfg.mres),) + A.shape[2:], dtype=A.dtype)
    for m in range(0, cfg.mmax + 1, cfg.mres):
        b = lm_index(cfg.lmax, cfg.mres, m, m)
        q[b:b + cfg.lmax - m + 1] = A[m:, m]
    return q


def unpack_lm(cfg: Config, q: np.ndarray) -> np.ndarray:
    q = np.asarray(q)
    A = np.zeros((cfg.lmax + 1, cfg.mmax + 1) + q.shape[1:], dtype=q.dtype)
    for m in range(0, cfg.mmax + 1, cfg.mres):
        b = lm_index(cfg.lmax, cfg.mres, m, m)
        A[m:, m] = q[b:b + cfg.lmax - m + 1]
    return A


def synthesis_packed(cfg: Config, q: np.ndarray, ltr: int | None = None) -> np.ndarray:
    """vec(synthesis(unpack_lm(q))) with degrees above ltr dropped."""
    return synthesis(cfg, unpack_lm(cfg, q), ltr=ltr).reshape(-1, order="F")


def analysis_packed(cfg: Config, v: np.ndarray, ltr: int | None = None) -> np.ndarray:
    return pack_lm(cfg, analysis(cfg, np.asarray(v).reshape(cfg.nlat, cfg.nlon, order="F"), ltr=ltr))


# ---------------------------------------------------------------------------
# Dense diagonal spectral operators, src/sphtor_transforms.jl:771-783 (δ = −l(l+1) S),
# :817-831 (S = −δ/(l(l+1))), :865-877 / :911-925 (vorticity/toroidal, same maps);
# ext/GPUCommon.jl:1501-1512 (laplacian_kernel!, the same map as the divergence).
# Entries with m % mres != 0 or l < max(1, m) become zero.
# ---------------------------------------------------------------------------

def _spectral_mask(cfg: Config, shape):
    l = np.arange(cfg.lmax + 1).reshape(-1, 1)
    m = np.arange(cfg.mmax + 1).reshape(1, -1)
    valid = (m % cfg.mres == 0) & (l >= np.maximum(1, m))
    return valid.reshape(valid.shape + (1,) * (len(shape) - 2)), l.reshape(l.shape + (1,) * (len(shape) - 2))


def neg_ll(cfg: Config, a: np.ndarray) -> np.ndarray:
    """divergence_from_spheroidal / vorticity_from_toroidal / laplacian: −l(l+1)·a."""
    a = np.asarray(a)
    valid, l = _spectral_mask(cfg, a.shape)
    ll = (l * (l + 1)).astype(a.real.dtype)
    out = np.empty_like(a)
    out.real = np.where(valid, -ll * a.real, 0)
    out.imag = np.where(valid, -ll * a.imag, 0)
    return out


def inv_neg_ll(cfg: Config, a: np.ndarray) -> np.ndarray:
    """spheroidal_from_divergence / toroidal_from_vorticity: −(a / (l(l+1))), componentwise."""
    a = np.asarray(a)
    valid, l = _spectral_mask(cfg, a.shape)
    ll = np.maximum(l * (l + 1), 1).astype(a.real.dtype)
    out = np.empty_like(a)
    out.real = np.where(valid, -(a.real / ll), 0)
    out.imag = np.where(valid, -(a.imag / ll), 0)
    return out


# ---------------------------------------------------------------------------
# Adjoints (Zygote convention g = 2 ∂L/∂ā), src/core_transforms.jl:477-652,
# src/sphtor_transforms.jl:385-452
# ---------------------------------------------------------------------------

def adjoint_synthesis(cfg: Config, ybar: np.ndarray, real_output: bool = True):
    Fb = np.fft.fft(np.asarray(ybar), axis=1)
    abar = np.zeros((cfg.lmax + 1, cfg.mmax + 1), dtype=np.complex128)
    phiadj = cfg.phi_inv_scale() / cfg.nlon
    for m in _mvals(cfg):
        wm = (1.0 if (m == 0 or not real_output) else 2.0) * phiadj
        P = plm_rows(cfg.x, cfg.lmax, m)
        abar[m:, m] = P[:, m:].T @ (wm * Fb[:, m])
    return abar if cfg.canonical else abar * cfg.scale_matrix()


def adjoint_analysis(cfg: Config, Abar: np.ndarray):
    """Complex spatial cotangent; the rrule projects it to real (ProjectTo)."""
    A = np.asarray(Abar, dtype=np.complex128)
    if not cfg.canonical:
        A = A / cfg.scale_matrix()
    F = np.zeros((cfg.nlat, cfg.nlon), dtype=np.complex128)
    phiadj = cfg.nlon * cfg.analysis_phi_scale()
    for m in _mvals(cfg):
        P = plm_rows(cfg.x, cfg.lmax, m)
        F[:, m] = (phiadj * cfg.w) * (P[:, m:] @ A[m:, m])
    return np.fft.ifft(F, axis=1)


def adjoint_synthesis_sphtor(cfg: Config, Vtb: np.ndarray, Vpb: np.ndarray, real_output: bool = True):
    Vtb = np.asarray(Vtb)
    Vpb = np.asarray(Vpb)
    if cfg.robert_form:
        st = cfg.sint()[:, None]
        Vtb = Vtb * st
        Vpb = Vpb * st
    Ft = np.fft.fft(Vtb, axis=1)
    Fp = np.fft.fft(Vpb, axis=1)
    Sb = np.zeros((cfg.lmax + 1, cfg.mmax + 1), dtype=np.complex128)
    Tb = np.zeros_like(Sb)
    phiadj = cfg.phi_inv_scale() / cfg.nlon
    for m in _mvals(cfg):
        lo = max(1, m)
        if lo > cfg.lmax:
            continue
        wm = (1.0 if (m == 0 or not real_output) else 2.0) * phiadj
        _, dP, Ps = plm_dtheta_rows(cfg.x, cfg.lmax, m)
        dY = dP[:, lo:]
        Ys = Ps[:, lo:]
        ft = Ft[:, m]
        fp = Fp[:, m]
        Sb[lo:, m] = wm * (dY.T @ ft - 1j * m * (Ys.T @ fp))
        Tb[lo:, m] = wm * (1j * m * (Ys.T @ ft) + dY.T @ fp)
    if not cfg.canonical:
        sc = cfg.scale_matrix()
        Sb = Sb * sc
        Tb = Tb * sc
    return Sb, Tb


def adjoint_analysis_sphtor(cfg: Config, Sbar: np.ndarray, Tbar: np.ndarray):
    S = np.asarray(Sbar, dtype=np.complex128)
    T = np.asarray(Tbar, dtype=np.complex128)
    if not cfg.canonical:
        sc = cfg.scale_matrix()
        S = S / sc
        T = T / sc
    Ft = np.zeros((cfg.nlat, cfg.nlon), dtype=np.complex128)
    Fp = np.zeros_like(Ft)
    phiadj = cfg.nlon * cfg.analysis_phi_scale()
    for m in _mvals(cfg):
        lo = max(1, m)
        if lo > cfg.lmax:
            continue
        _, dP, Ps = plm_dtheta_rows(cfg.x, cfg.lmax, m)
        ls = np.arange(lo, cfg.lmax + 1)
        c = 1.0 / (ls * (ls + 1.0))
        s = S[lo:, m] * c
        t = T[lo:, m] * c
        dY = dP[:, lo:]
        Ys = Ps[:, lo:]
        Ft[:, m] = phiadj * cfg.w * (dY @ s - 1j * m * (Ys @ t))
        Fp[:, m] = phiadj * cfg.w * (1j * m * (Ys @ s) + dY @ t)
    vt = np.fft.ifft(Ft, axis=1)
    vp = np.fft.ifft(Fp, axis=1)
    if cfg.robert_form:
        st = cfg.sint()
        inv = np.where(st > 0, 1.0 / np.where(st > 0, st, 1.0), 1.0)[:, None]
        vt = vt * inv
        vp = vp * inv
    return vt, vp


# ---------------------------------------------------------------------------
# Batched forms: trailing field index, P̄ rows shared across fields
# (src/batch_transforms.jl:372-553)
# ---------------------------------------------------------------------------

def synthesis_batch(cfg: Config, alm: np.ndarray, real_output: bool = True):
    a = np.asarray(alm, dtype=np.complex128)
    if not cfg.canonical:
        a = a * cfg.scale_matrix()[:, :, None]
    nf = a.shape[2]
    F = np.zeros((cfg.nlat, cfg.nlon, nf), dtype=np.complex128)
    for m in _mvals(cfg):
        P = plm_rows(cfg.x, cfg.lmax, m)
        F[:, m, :] = cfg.phi_inv_scale() * (P[:, m:] @ a[m:, m, :])
    if real_output:
        for m in range(1, cfg.mmax + 1):
            F[:, cfg.nlon - m, :] = np.conj(F[:, m, :])
    f = np.fft.ifft(F, axis=1)
    return f.real.copy() if real_output else f


def analysis_batch(cfg: Config, f: np.ndarray):
    F = np.fft.fft(np.asarray(f), axis=1)
    nf = F.shape[2]
    alm = np.zeros((cfg.lmax + 1, cfg.mmax + 1, nf), dtype=np.complex128)
    sc = cfg.analysis_phi_scale()
    for m in _mvals(cfg):
        P = plm_rows(cfg.x, cfg.lmax, m)
        alm[m:, m, :] = ((cfg.w * sc)[:, None] * P[:, m:]).T @ F[:, m, :]
    if not cfg.canonical:
        alm = alm / cfg.scale_matrix()[:, :, None]
        for m in range(cfg.mmax + 1):
            alm[:m, m, :] = 0
    return alm


def synthesis_sphtor_batch(cfg, S, T, real_output=True):
    outs = [synthesis_sphtor(cfg, S[:, :, k], T[:, :, k], real_output) for k in range(S.shape[2])]
    return np.stack([o[0] for o in outs], axis=2), np.stack([o[1] for o in outs], axis=2)


def analysis_sphtor_batch(cfg, Vt, Vp):
    outs = [analysis_sphtor(cfg, Vt[:, :, k], Vp[:, :, k]) for k in range(Vt.shape[2])]
    return np.stack([o[0] for o in outs], axis=2), np.stack([o[1] for o in outs], axis=2)


def balanced_m_order(mmax: int, mres: int = 1) -> list[int]:
    """Zig-zag m schedule (``src/buffer_utils.jl:16-25``)."""
    n = mmax // mres + 1
    return [((i // 2) if i % 2 == 0 else (n - 1) - i // 2) * mres for i in range(n)]


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)
