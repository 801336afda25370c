"""Uneven batches: many independent mixed-precision scalar roundtrips of different sizes.

Each member has its own configuration (lmax, Gauss grid, nlon) and 1..8 fields. The
library runs all members' tiles in one persistent launch per stage (B packing,
order-GEMM synthesis, FFT synthesis, FFT analysis, order-GEMM analysis), captured once into a
CUDA graph and replayed (``shtb_group_*`` in ``include/shtb200.h``). Results equal
the per-member ``synthesis_batch`` / ``analysis_batch`` calls with
``precision="mixed"`` bit for bit.

No counterpart in the reference: SHTnsKit.jl runs one configuration per call
(src/batch_transforms.jl); this is the batching layer a training loop over mixed
resolutions would put around it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .config import SHTConfig
from .transforms import julia_empty


def smooth_nlon(lmax: int) -> int:
    """Smallest 2^a 3^b 5^c >= 2 (lmax + 1)."""
    n = 2 * (lmax + 1)
    while True:
        k = n
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return n
        n += 1


class UnevenBatch:
    """A group of transforms with their own configurations, run as one graph launch.

    ``cfgs``: list of :class:`SHTConfig` (mres = 1, lcap = lmax); ``nfields``: fields
    per member (int or list). Device buffers are allocated here in the Julia layout:
    ``alm_in[t]`` / ``alm_out[t]`` of shape (lmax+1, mmax+1, nf) complex64 and
    ``grid[t]`` of shape (nlat, nlon, nf) float32.
    """

    def __init__(self, cfgs: list[SHTConfig], nfields=1, device_index: int = 0):
        self.cfgs = list(cfgs)
        n = len(self.cfgs)
        self.nf = [nfields] * n if isinstance(nfields, int) else list(nfields)
        self.device_index = device_index
        dev = torch.device("cuda", device_index)
        lib = _lib.load()
        plans = [c.plan(device_index) for c in self.cfgs]
        self._plans = plans
        arr = (ctypes.c_void_p * n)(*[p.handle for p in plans])
        nfa = (ctypes.c_int * n)(*self.nf)
        h = ctypes.c_void_p()
        with torch.cuda.device(device_index):
            _lib.check(lib.shtb_group_create(ctypes.byref(h), arr, n, nfa), "group_create")
        self.handle = h.value
        self.alm_in = [julia_empty((c.lmax + 1, c.mmax + 1, k), torch.complex64, dev) for c, k in zip(self.cfgs, self.nf)]
        self.alm_out = [julia_empty((c.lmax + 1, c.mmax + 1, k), torch.complex64, dev) for c, k in zip(self.cfgs, self.nf)]
        self.grid = [julia_empty((c.nlat, c.nlon, k), torch.float32, dev) for c, k in zip(self.cfgs, self.nf)]
        for t in self.alm_in + self.alm_out + self.grid:
            t.zero_()
        ptrs = lambda ts: (ctypes.c_void_p * n)(*[t.data_ptr() for t in ts])  # noqa: E731
        with torch.cuda.device(device_index):
            _lib.check(lib.shtb_group_bind(self.handle, ptrs(self.alm_in), ptrs(self.grid), ptrs(self.alm_out)),
                       "group_bind")

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device_index).cuda_stream

    def roundtrip(self) -> None:
        """alm_in -> grid -> alm_out for every member: one CUDA graph launch on the current stream."""
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.load().shtb_group_roundtrip(self.handle, self._stream()), "group_roundtrip")

    def launch(self, op: int = -1) -> None:
        """The same stages as direct launches (op: SHTB_OP_SYNTHESIS, SHTB_OP_ANALYSIS or -1)."""
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.load().shtb_group_launch(self.handle, op, self._stream()), "group_launch")

    def autotune(self) -> tuple[int, int, int]:
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.load().shtb_group_autotune(self.handle, self._stream()), "group_autotune")
        return self.config()

    def config(self) -> tuple[int, int, int]:
        """(FFT latitude pairs per CTA, FFT CTAs, GEMM CTAs)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.load().shtb_group_config(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                   "group_config")
        return a.value, b.value, c.value

    def latencies_ns(self) -> np.ndarray:
        """Per-member completion time of the last roundtrip, ns after its start."""
        torch.cuda.synchronize(self.device_index)
        out = np.zeros(len(self.cfgs), dtype=np.uint64)
        _lib.check(_lib.load().shtb_group_latency_ns(self.handle, out.ctypes.data), "group_latency_ns")
        return out

    def status(self) -> None:
        for p in self._plans:
            p.status()

    def close(self) -> None:
        if getattr(self, "handle", None):
            _lib.load().shtb_group_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
