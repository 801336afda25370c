"""CPU: the oracle's dense diagonal spectral operators against the reference's own
test cases for them (test/parity/operators.jl:92-131, :205-216; test/parity/sphtor_full.jl:
290-340): mres = 2 with adversarial storage in forbidden columns, l = 0 cleared, the
Laplacian kernel on a dense ramp equal to the divergence map, and the inverse recovering
the input on the valid entries."""
import numpy as np

from oracle import sht_oracle as so


def test_divergence_map_and_inverse_mres2():
    cfg = so.create_gauss_config(6, 8, mres=2)
    rng = np.random.default_rng(0xD1A6)
    a = (rng.standard_normal((7, 7)) + 1j * rng.standard_normal((7, 7))).astype(np.complex64)
    d = so.neg_ll(cfg, a)
    assert d.dtype == np.complex64
    assert np.all(d[:, 1] == 0) and d[0, 0] == 0          # column m = 1 is forbidden with mres = 2
    for m in range(0, 7, 2):
        for l in range(max(1, m), 7):
            assert d[l, m] == np.complex64(-(l * (l + 1))) * a[l, m]
    back = so.inv_neg_ll(cfg, d)
    expected = a.copy()
    for m in range(7):
        for l in range(7):
            if m % 2 or l < max(1, m):
                expected[l, m] = 0
    assert np.allclose(back, expected, rtol=1e-6, atol=0)


def test_laplacian_ramp_equals_divergence():
    cfg = so.create_gauss_config(5, 6, mmax=4)
    dense = (np.arange(1, 6 * 5 + 1).reshape(5, 6).T).astype(np.complex128)   # CT.(1:N), column-major
    lap = so.neg_ll(cfg, dense)
    for m in range(5):
        for l in range(6):
            want = -(l * (l + 1)) * dense[l, m] if l >= max(1, m) else 0
            assert lap[l, m] == want


def test_batched_trailing_field_axis():
    cfg = so.create_gauss_config(9, 10)
    rng = np.random.default_rng(3)
    a = rng.standard_normal((10, 10, 3)) + 1j * rng.standard_normal((10, 10, 3))
    d = so.neg_ll(cfg, a)
    for k in range(3):
        assert np.array_equal(d[:, :, k], so.neg_ll(cfg, a[:, :, k]))
    assert np.array_equal(so.inv_neg_ll(cfg, a)[:, :, 1], so.inv_neg_ll(cfg, a[:, :, 1]))


def test_packed_lm_layout():
    """LM_index walks the m blocks of l = m..lmax contiguously (src/layout.jl:143-162), and
    pack/unpack invert each other on the stored entries."""
    for lmax, mmax, mres in ((4, 4, 2), (9, 6, 3), (12, 12, 1)):
        cfg = so.create_gauss_config(lmax, lmax + 2, mmax=mmax, mres=mres)
        idx = [so.lm_index(lmax, mres, l, m) for m in range(0, mmax + 1, mres) for l in range(m, lmax + 1)]
        assert idx == list(range(so.nlm_calc(lmax, mmax, mres)))
        rng = np.random.default_rng(lmax)
        A = rng.standard_normal((lmax + 1, mmax + 1)) + 1j * rng.standard_normal((lmax + 1, mmax + 1))
        q = so.pack_lm(cfg, A)
        back = so.unpack_lm(cfg, q)
        for m in range(mmax + 1):
            for l in range(lmax + 1):
                assert back[l, m] == (A[l, m] if (m % mres == 0 and l >= m) else 0)
    assert so.lm_index(4, 2, 2, 2) == 5 and so.lm_index(4, 2, 4, 4) == 8


def test_packed_transforms_oracle_roundtrip():
    cfg = so.create_gauss_config(15, 16)
    rng = np.random.default_rng(8)
    A = rng.standard_normal((16, 16)) + 1j * rng.standard_normal((16, 16))
    A = np.tril(A)
    A[:, 0] = A[:, 0].real
    q = so.pack_lm(cfg, A)
    v = so.synthesis_packed(cfg, q)
    assert v.shape == (16 * cfg.nlon,)
    assert np.allclose(so.analysis_packed(cfg, v), q, rtol=0, atol=1e-12)


def test_mirror_lm_index_matches_oracle_and_rejects():
    """The host mirror's LM_index / nlm_calc (no GPU) against the oracle, and the reference's
    argument errors (src/layout.jl:143-162)."""
    import pytest
    import shtb200 as sht
    for lmax, mmax, mres in ((7, 7, 1), (10, 8, 2), (12, 9, 3)):
        assert sht.nlm_calc(lmax, mmax, mres) == so.nlm_calc(lmax, mmax, mres)
        for m in range(0, mmax + 1, mres):
            for l in range(m, lmax + 1):
                assert sht.LM_index(lmax, mres, l, m) == so.lm_index(lmax, mres, l, m)
    assert sht.nlm_calc(3, 5, 1) == 0
    for bad in ((4, 2, 3, 1), (4, 1, 1, 2), (4, 1, 5, 1), (4, 1, -1, -1)):
        with pytest.raises(sht.ArgumentError):
            sht.LM_index(*bad)
