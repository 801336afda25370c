"""ctypes wrapper of ``liboracle.so`` (the C restatement in ``sht_oracle.c``).

TEST INFRASTRUCTURE AND CPU BASELINE ONLY (see ``sht_oracle.c``)."""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "liboracle.so"
_lib = None


def load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(LIB))
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        _lib.oracle_synthesis_batch.argtypes = [I, I, I, I, I, P, P, P, I, D, I]
        _lib.oracle_analysis_batch.argtypes = [I, I, I, I, I, P, P, P, P, I, D, I]
        _lib.oracle_max_threads.restype = I
    return _lib


def max_threads() -> int:
    return load().oracle_max_threads()


def synthesis_batch(cfg, alm: np.ndarray, nthreads: int = 0) -> np.ndarray:
    """cfg: oracle Config (canonical). alm (lmax+1, mmax+1, nf) complex -> (nlat, nlon, nf)."""
    a = np.asfortranarray(alm, dtype=np.complex128)
    nf = a.shape[2]
    f = np.zeros((cfg.nlat, cfg.nlon, nf), order="F")
    load().oracle_synthesis_batch(cfg.lmax, cfg.mmax, cfg.mres, cfg.nlat, cfg.nlon, cfg.x.ctypes.data,
                                  a.ctypes.data, f.ctypes.data, nf, cfg.phi_inv_scale(), nthreads)
    return f


def analysis_batch(cfg, f: np.ndarray, nthreads: int = 0) -> np.ndarray:
    g = np.asfortranarray(f, dtype=np.float64)
    nf = g.shape[2]
    a = np.zeros((cfg.lmax + 1, cfg.mmax + 1, nf), dtype=np.complex128, order="F")
    load().oracle_analysis_batch(cfg.lmax, cfg.mmax, cfg.mres, cfg.nlat, cfg.nlon, cfg.x.ctypes.data,
                                 cfg.w.ctypes.data, g.ctypes.data, a.ctypes.data, nf, cfg.analysis_phi_scale(),
                                 nthreads)
    return a
