"""CPU checks of the fp16x3 numerics of the mixed path (no GPU).

The tensor-core GEMMs multiply f16 hi/lo splits of both operands (hi*hi + hi*lo + lo*hi,
FP32 accumulation). f16 has 5 exponent bits, so the kernels scale by powers of two first:
the P table by 2^s for the whole plan (csrc/mixed.cu, f16_table_exp), every B row by 2^e
so that its largest magnitude lies in [2^14, 2^15). These tests restate those rules in
numpy and check (1) that the table scale keeps every P value of the oracle below 2^15 and
(2) that the split products meet the 1e-6 bar across rows of very different magnitude,
which plain f16 without the row scales does not.
"""
import numpy as np
import pytest

from oracle import sht_oracle as so


def table_exp(lmax):
    """The largest s <= 14 with 2^s sqrt(2 (2L+1) / (4 pi)) <= 2^15, L = lmax + 1."""
    q = 2 * (lmax + 1) + 1
    s = 14
    while s > 0 and (q << (2 * s)) > 6746518852:   # floor(2^31 pi)
        s -= 1
    return s


def row_exp(x32):
    """Power of two bringing the row's largest magnitude into [2^14, 2^15), at most 100."""
    bits = np.abs(x32).view(np.uint32).max(initial=np.uint32(0))
    return min(141 - int(bits >> 23), 100)


def split16(x32):
    """hi = f16(x) rounded to nearest, lo = f16(x - hi); x - hi is exact in FP32."""
    hi = x32.astype(np.float16)
    lo = (x32 - hi.astype(np.float32)).astype(np.float16)
    return hi.astype(np.float32), lo.astype(np.float32)


def fp16x3_dot(p32, b32, s, chunk=64):
    """sum_k p[k] b[k] as the GEMM forms it: P pre-scaled by 2^s, B scaled per chunk by 2^e,
    cross terms then hi*hi per chunk in FP32, chunk sums promoted with 2^-(e+s)."""
    acc = np.float32(0.0)
    for k0 in range(0, p32.size, chunk):
        a = np.ldexp(p32[k0:k0 + chunk], s).astype(np.float32)
        b = b32[k0:k0 + chunk]
        e = row_exp(b)
        ah, al = split16(a)
        bh, bl = split16(np.ldexp(b, e).astype(np.float32))
        part = np.float32(np.sum(ah * bl, dtype=np.float32) + np.sum(al * bh, dtype=np.float32))
        part = np.float32(part + np.sum(ah * bh, dtype=np.float32))
        acc = np.float32(acc + np.float32(np.ldexp(np.float64(part), -(e + s))))
    return float(acc)


@pytest.mark.parametrize("lmax", [15, 63, 255])
def test_table_scale_bounds_every_p_value(lmax):
    x, _ = so.gauss_legendre(lmax + 1)
    s = table_exp(lmax)
    pmax = max(np.abs(so.plm_rows(x, lmax + 1, m)).max() for m in range(lmax + 1))
    assert pmax * 2.0 ** s < 2.0 ** 15   # f16 maximum 65504: hi never overflows


@pytest.mark.parametrize("lmax", [511, 1023, 2047, 4095])
def test_table_scale_large_lmax(lmax):
    x, _ = so.gauss_legendre(min(lmax + 1, 1024))
    s = table_exp(lmax)
    assert s >= 8   # the f16 subnormal floor stays below 2^-33 of P
    for m in (0, 1, lmax // 2):
        assert np.abs(so.plm_rows(x, lmax + 1, m)).max() * 2.0 ** s < 2.0 ** 15
    # |P_l^m| <= sqrt((2l+1)/(4 pi)) for every m (addition theorem): the bound the exponent uses
    assert np.sqrt((2 * (lmax + 1) + 1) / (4 * np.pi)) * np.sqrt(2) * 2.0 ** s <= 2.0 ** 15


def test_fp16x3_products_across_magnitudes():
    rng = np.random.default_rng(1)
    lmax, m = 255, 3
    x, _ = so.gauss_legendre(lmax + 1)
    P = so.plm_rows(x, lmax + 1, m)[:, m::2].astype(np.float32)   # one parity, K = degrees
    s = table_exp(lmax)
    for scale in (1.0, 1e25, 1e-25, 3e-30):
        b = (rng.standard_normal(P.shape[1]) / (1.0 + np.arange(P.shape[1]))).astype(np.float32) * np.float32(scale)
        b = b.astype(np.float32)
        for i in range(0, P.shape[0], 37):
            ref = float(np.dot(P[i].astype(np.float64), b.astype(np.float64)))
            got = fp16x3_dot(P[i], b, s)
            mag = float(np.sum(np.abs(P[i].astype(np.float64) * b.astype(np.float64))))
            assert abs(got - ref) <= 1e-6 * mag, (scale, i)


def test_unscaled_f16_fails_for_small_rows():
    """Without the row scale a row of magnitude 1e-10 underflows f16 and loses everything."""
    rng = np.random.default_rng(2)
    b = (rng.standard_normal(64) * 1e-10).astype(np.float32)
    bh, bl = split16(b)
    assert np.abs(bh + bl - b).max() > 0.5 * np.abs(b).max()
    e = row_exp(b)
    sh, sl = split16(np.ldexp(b, e).astype(np.float32))
    back = np.ldexp(sh.astype(np.float64) + sl, -e)
    assert np.abs(back - b).max() <= 2.0 ** -21 * np.abs(b).max()


def test_row_exp_edges():
    assert row_exp(np.zeros(8, np.float32)) == 100
    assert row_exp(np.array([1.0], np.float32)) == 14
    assert row_exp(np.array([np.float32(3.4e38)], np.float32)) == 141 - 254
    v = np.array([0.75, -1.5], np.float32)
    e = row_exp(v)
    assert 2.0 ** 14 <= 1.5 * 2.0 ** e < 2.0 ** 15
