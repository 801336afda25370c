"""CPU: host mirror logic — configuration validation, scale conventions, layouts."""
import math
import os

import numpy as np
import pytest
import torch

import shtb200 as sht
from shtb200 import transforms as T
from oracle import sht_oracle as so


def test_config_matches_reference_rules():
    cfg = sht.create_gauss_config(31, 32)
    assert cfg.nlon == 64 and cfg.mmax == 31 and cfg.nlm == 32 * 33 // 2
    assert cfg.phi_inv_scale() == 64.0
    assert abs(cfg.analysis_phi_scale() - 2 * math.pi / 64) < 1e-16
    for bad in [dict(lmax=4, nlat=4), dict(lmax=4, nlat=5, nlon=8), dict(lmax=4, nlat=5, mmax=5)]:
        with pytest.raises(sht.ArgumentError):
            sht.create_gauss_config(bad.pop("lmax"), bad.pop("nlat"), **bad)


def test_phi_scale_env(monkeypatch):
    cfg = sht.create_gauss_config(7, 8)
    monkeypatch.setenv("SHTNSKIT_PHI_SCALE", "quad")
    assert abs(cfg.phi_inv_scale() - cfg.nlon / (2 * math.pi)) < 1e-12
    assert abs(cfg.analysis_phi_scale() - 4 * math.pi ** 2 / cfg.nlon) < 1e-14


@pytest.mark.parametrize("kw", [dict(norm="schmidt"), dict(real_norm=True), dict(cs_phase=False),
                                dict(norm="fourpi", real_norm=True, cs_phase=False)])
def test_scale_matrix_matches_oracle(kw):
    cfg = sht.create_gauss_config(6, 8, **kw)
    ocfg = so.create_gauss_config(6, 8, **kw)
    s, so_s = cfg.scale_matrix(), ocfg.scale_matrix()
    for m in range(7):
        assert np.allclose(s[m:, m], so_s[m:, m], rtol=0, atol=0)
    assert sht.create_gauss_config(6, 8).scale_matrix() is None


def test_julia_layout_helpers():
    t = T.julia_empty((3, 4, 5), torch.float64, "cpu")
    assert t.stride() == (1, 3, 12) and T.is_julia_dense(t)
    a = np.arange(60.0).reshape(3, 4, 5)
    h = T.to_host(torch.from_numpy(np.asfortranarray(a)))
    assert np.array_equal(h, a)


def test_device_markers():
    assert isinstance(sht.on_device(np.zeros(3)), sht.CPU)
    assert isinstance(sht.on_device(torch.zeros(3)), sht.CPU)


def test_transform_arguments_rejected_before_device():
    """The mirror raises the reference's errors for bad arguments before any device work."""
    cfg = sht.create_gauss_config(15, 16, nlon=32)
    alm = np.zeros((16, 16), np.complex64)
    with pytest.raises(sht.ArgumentError, match="precision must be 'fp64' or 'mixed'"):
        sht.synthesis(cfg, alm, precision="bf16")
    with pytest.raises(sht.ArgumentError, match="lcap"):
        sht.synthesis(cfg, alm, lcap=16, precision="mixed")
    with pytest.raises(sht.ArgumentError, match="use_rfft=true implies real_output"):
        sht.synthesis(cfg, alm, real_output=False, use_rfft=True)
    with pytest.raises(sht.BackendUnavailableError):
        sht.synthesis(cfg, alm, real_output=False)
    with pytest.raises(sht.DimensionMismatch):
        sht.synthesis(cfg, np.zeros((16, 16, 2), np.complex64), precision="mixed")
    with pytest.raises(sht.ArgumentError, match="precision"):
        sht.analysis_batch(cfg, np.zeros((16, 32, 2), np.float32), precision="tf32")
