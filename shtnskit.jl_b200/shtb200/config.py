"""Host mirror of SHTnsKit's ``SHTConfig`` for Gauss-Legendre grids.

Mirrors ``create_gauss_config`` / ``create_gauss_fly_config`` (src/config.jl:633-701),
``_validate_spectral_layout`` (src/config.jl:465-481), the normalization scale
``coefficient_scale_to_canonical`` (src/normalization.jl:142-147) and the φ-scale
rules ``phi_inv_scale`` / ``_analysis_phi_scale`` (src/SHTnsKit.jl:128-177).
Gauss nodes come from the library's C++ ``shtb_gauss_nodes``.

A config owns one device plan per CUDA device, built on first use and cached
(the reference caches its device tables per config, ext/SHTnsKitGPUExt.jl:495-518).
"""
from __future__ import annotations

import ctypes
import math
import os
import threading
import weakref

import numpy as np

from . import _lib
from ._lib import ArgumentError


def _default_nlon(lmax: int) -> int:
    """Next even integer >= 2*lmax+1 (src/config.jl:76-80)."""
    n = 2 * lmax + 1
    return n + (n & 1)


def validate_spectral_layout(lmax: int, mmax: int, mres: int, nlat: int, nlon: int) -> None:
    if lmax < 0:
        raise ArgumentError(f"lmax must be ≥ 0, got {lmax}")
    if mmax < 0:
        raise ArgumentError(f"mmax must be ≥ 0, got {mmax}")
    if mmax > lmax:
        raise ArgumentError(f"mmax must be ≤ lmax, got mmax={mmax}, lmax={lmax}")
    if mres < 1:
        raise ArgumentError(f"mres must be ≥ 1, got {mres}")
    if nlat < 1:
        raise ArgumentError(f"nlat must be ≥ 1, got {nlat}")
    if nlat < lmax + 1:
        raise ArgumentError(f"Gauss–Legendre quadrature requires nlat ≥ lmax+1, got nlat={nlat} and lmax={lmax}")
    if nlon < 2 * mmax + 1:
        raise ArgumentError(
            f"nlon must be ≥ 2*mmax+1 = {2 * mmax + 1} to resolve every azimuthal order, got nlon={nlon}")


def gauss_nodes(n: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Legendre nodes (north pole first) and weights from the C ABI."""
    lib = _lib.load()
    x = np.empty(n, dtype=np.float64)
    w = np.empty(n, dtype=np.float64)
    _lib.check(lib.shtb_gauss_nodes(n, x.ctypes.data, w.ctypes.data), "gauss_nodes")
    return x, w


def _norm_scale_from_orthonormal(l: int, norm: str) -> float:
    if norm == "orthonormal":
        return 1.0
    if norm == "fourpi":
        return math.sqrt(4 * math.pi)
    if norm == "schmidt":
        return math.sqrt(4 * math.pi / (2 * l + 1))
    raise ArgumentError(f"Unsupported normalization: {norm}")


class SHTConfig:
    """Gauss grid configuration; field names follow the reference's ``SHTConfig``."""

    def __init__(self, lmax, nlat, mmax, mres, nlon, norm="orthonormal", cs_phase=True, real_norm=False,
                 robert_form=False, phi_scale="dft", on_the_fly=False):
        validate_spectral_layout(lmax, mmax, mres, nlat, nlon)
        if norm not in ("orthonormal", "fourpi", "schmidt"):
            raise ArgumentError(f"Unsupported normalization: {norm}")
        self.lmax, self.nlat, self.mmax, self.mres, self.nlon = lmax, nlat, mmax, mres, nlon
        self.norm, self.cs_phase, self.real_norm = norm, bool(cs_phase), bool(real_norm)
        self.robert_form = bool(robert_form)
        self.phi_scale = phi_scale
        self.on_the_fly = on_the_fly
        self.grid_type = "gauss"
        self.x, self.w = gauss_nodes(nlat)
        self.cphi = 2 * math.pi / nlon
        self._plans: dict = {}
        self._plan_lock = threading.Lock()
        self._finalizer = weakref.finalize(self, _destroy_plans, self._plans)

    # --- derived quantities -------------------------------------------------
    @property
    def nlm(self) -> int:
        return sum(self.lmax - m + 1 for m in range(0, self.mmax + 1, self.mres))

    @property
    def canonical(self) -> bool:
        return self.norm == "orthonormal" and not self.real_norm and self.cs_phase

    def phi_inv_scale(self) -> float:
        mode = os.environ.get("SHTNSKIT_PHI_SCALE", "")
        if mode == "quad":
            return self.nlon / (2 * math.pi)
        if mode == "dft":
            return float(self.nlon)
        return self.nlon / (2 * math.pi) if self.phi_scale == "quad" else float(self.nlon)

    def analysis_phi_scale(self) -> float:
        return self.cphi * self.nlon / self.phi_inv_scale()

    def scale_matrix(self) -> np.ndarray | None:
        """s[l, m] with a_canonical = s * a_configured, column-major (lmax+1, mmax+1); None if canonical."""
        if self.canonical:
            return None
        s = np.ones((self.lmax + 1, self.mmax + 1))
        for m in range(self.mmax + 1):
            for l in range(m, self.lmax + 1):
                v = _norm_scale_from_orthonormal(l, self.norm)
                if self.real_norm and m > 0:
                    v *= 1.0 / math.sqrt(2.0)
                if not self.cs_phase:
                    v *= (-1.0) ** m
                s[l, m] = v
        return s

    # --- device plan ---------------------------------------------------------
    def plan(self, device_index: int) -> "Plan":
        key = (device_index, self.phi_inv_scale())
        with self._plan_lock:
            p = self._plans.get(key)
            if p is None:
                p = Plan(self, device_index)
                self._plans[key] = p
            return p

    def clear_plans(self) -> None:
        with self._plan_lock:
            _destroy_plans(self._plans)

    def __repr__(self):
        return (f"SHTConfig(lmax={self.lmax}, mmax={self.mmax}, mres={self.mres}, nlat={self.nlat}, "
                f"nlon={self.nlon}, grid=gauss, norm={self.norm}, cs_phase={self.cs_phase}, "
                f"real_norm={self.real_norm}, robert_form={self.robert_form})")


def _destroy_plans(plans: dict) -> None:
    for p in list(plans.values()):
        p.destroy()
    plans.clear()


class Plan:
    """Owns one ``shtb_plan`` on one device."""

    def __init__(self, cfg: SHTConfig, device_index: int):
        import torch

        lib = _lib.load()
        self.device_index = device_index
        self.cfg_dims = (cfg.lmax, cfg.mmax, cfg.mres, cfg.nlat, cfg.nlon)
        sc = cfg.scale_matrix()
        sc_arr = None if sc is None else np.asfortranarray(sc)
        handle = ctypes.c_void_p()
        with torch.cuda.device(device_index):
            rc = lib.shtb_plan_create(
                ctypes.byref(handle), cfg.lmax, cfg.mmax, cfg.mres, cfg.nlat, cfg.nlon,
                cfg.x.ctypes.data, cfg.w.ctypes.data,
                None if sc_arr is None else sc_arr.ctypes.data,
                cfg.phi_inv_scale(), cfg.analysis_phi_scale(), 1 if cfg.robert_form else 0)
        _lib.check(rc, "plan_create")
        self.handle = handle.value
        self._alive = True

    def workspace_bytes(self, op: int, nfields: int, dtype: int, precision: int) -> int:
        return int(_lib.load().shtb_workspace_bytes(self.handle, op, nfields, dtype, precision))

    def table_bytes(self) -> int:
        return int(_lib.load().shtb_plan_table_bytes(self.handle))

    def status(self) -> None:
        """Raise BackendUnavailableError if a kernel of this plan gave up a bounded device wait."""
        import torch

        with torch.cuda.device(self.device_index):
            _lib.check(_lib.load().shtb_plan_status(self.handle), "plan_status")

    def destroy(self) -> None:
        if getattr(self, "_alive", False):
            self._alive = False
            try:
                import torch

                with torch.cuda.device(self.device_index):
                    _lib.load().shtb_plan_destroy(self.handle)
            except Exception:  # interpreter shutdown
                pass


def create_gauss_config(lmax: int, nlat: int, *, mmax: int | None = None, mres: int = 1, nlon: int | None = None,
                        norm: str = "orthonormal", cs_phase: bool = True, real_norm: bool = False,
                        robert_form: bool = False) -> SHTConfig:
    mmax = lmax if mmax is None else mmax
    nlon = _default_nlon(lmax) if nlon is None else nlon
    return SHTConfig(lmax, nlat, mmax, mres, nlon, norm, cs_phase, real_norm, robert_form, "dft")


def create_gauss_fly_config(lmax: int, nlat: int, **kw) -> SHTConfig:
    cfg = create_gauss_config(lmax, nlat, **kw)
    cfg.on_the_fly = True
    return cfg
