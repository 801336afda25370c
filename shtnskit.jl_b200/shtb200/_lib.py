"""ctypes binding of ``libshtb200.so`` (the C ABI declared in ``include/shtb200.h``).

The library is built in-tree next to this file. Importing this module never
falls back to anything else: if the library is missing or a symbol is absent,
``load()`` raises :class:`BackendUnavailableError`.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libshtb200.so"

SHTB_OK = 0
SHTB_ERR_BAD_ARG = -1
SHTB_ERR_BAD_SHAPE = -2
SHTB_ERR_ALIGN = -3
SHTB_ERR_OOM = -4
SHTB_ERR_CUDA = -5
SHTB_ERR_TIMEOUT = -6
SHTB_ERR_UNSUPPORTED = -7
SHTB_ERR_WORKSPACE = -8

SHTB_F64 = 0
SHTB_F32 = 1
SHTB_PREC_FP64 = 0
SHTB_PREC_MIXED = 1

SHTB_OP_SYNTHESIS = 0
SHTB_OP_ANALYSIS = 1
SHTB_OP_SYNTHESIS_SPHTOR = 2
SHTB_OP_ANALYSIS_SPHTOR = 3

SHTB_SPEC_NEG_LL = 0
SHTB_SPEC_INV_NEG_LL = 1


class BackendUnavailableError(RuntimeError):
    """Mirror of SHTnsKit's ``BackendUnavailableError(operation, detail)`` (src/devices.jl:20-26)."""

    def __init__(self, operation: str, detail: str):
        super().__init__(f"GPU backend unavailable for `{operation}`: {detail}")
        self.operation = operation
        self.detail = detail


class DimensionMismatch(ValueError):
    """Mirror of Julia's ``DimensionMismatch``."""


class ArgumentError(ValueError):
    """Mirror of Julia's ``ArgumentError``."""


# (name, restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t
SIGNATURES = {
    "shtb_version": (_I, []),
    "shtb_last_error": (ctypes.c_char_p, []),
    "shtb_gauss_nodes": (_I, [_I, _P, _P]),
    "shtb_plan_create": (_I, [ctypes.POINTER(_P), _I, _I, _I, _I, _I, _P, _P, _P, _D, _D, _I]),
    "shtb_plan_destroy": (_I, [_P]),
    "shtb_plan_table_bytes": (_SZ, [_P]),
    "shtb_plan_status": (_I, [_P]),
    "shtb_plan_debug_waits": (_I, [_P, ctypes.c_uint64, _I]),
    "shtb_workspace_bytes": (_SZ, [_P, _I, _I, _I, _I]),
    "shtb_synthesis": (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_analysis": (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_synthesis_cplx": (_I, [_P, _P, _P, _I, _I, _P, _SZ, _P]),
    "shtb_analysis_cplx": (_I, [_P, _P, _P, _I, _I, _P, _SZ, _P]),
    "shtb_synthesis_sphtor": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_analysis_sphtor": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_synthesis_packed": (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_analysis_packed": (_I, [_P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_synthesis_divvort": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_analysis_divvort": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _SZ, _P]),
    "shtb_spectral_op": (_I, [_P, _I, _P, _P, _I, _I, _P]),
    "shtb_synthesis_adjoint": (_I, [_P, _P, _P, _I, _P, _SZ, _P]),
    "shtb_analysis_adjoint": (_I, [_P, _P, _P, _I, _P, _SZ, _P]),
    "shtb_synthesis_sphtor_adjoint": (_I, [_P, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "shtb_analysis_sphtor_adjoint": (_I, [_P, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "shtb_synthesis_noalloc": (_I, [_P, _P, _P, _I, _I, _P]),
    "shtb_group_create": (_I, [ctypes.POINTER(_P), _P, _I, _P]),
    "shtb_group_destroy": (_I, [_P]),
    "shtb_group_bind": (_I, [_P, _P, _P, _P]),
    "shtb_group_roundtrip": (_I, [_P, _P]),
    "shtb_group_launch": (_I, [_P, _I, _P]),
    "shtb_group_autotune": (_I, [_P, _P]),
    "shtb_group_config": (_I, [_P, _P, _P, _P]),
    "shtb_group_latency_ns": (_I, [_P, _P]),
    "shtb_launch_count": (ctypes.c_uint64, [_I]),
    "shtb_profile_enable": (_I, [_I]),
    "shtb_profile_read": (_I, [_I, ctypes.c_char_p, _P, _P]),
}

_lib = None
_lock = threading.Lock()


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load the library once; raise BackendUnavailableError when it is not built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise BackendUnavailableError("load", f"{p.name} is not built; run __graft_entry__.build() or make -C csrc")
        try:
            lib = ctypes.CDLL(str(p))
        except OSError as e:
            raise BackendUnavailableError("load", f"cannot load {p}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            try:
                fn = getattr(lib, name)
            except AttributeError as e:
                raise BackendUnavailableError("load", f"symbol {name} missing from {p.name}") from e
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc: int, operation: str) -> None:
    """Map a status code to the exception the reference would throw."""
    if rc == SHTB_OK:
        return
    msg = load().shtb_last_error().decode(errors="replace")
    if rc == SHTB_ERR_BAD_SHAPE:
        raise DimensionMismatch(msg)
    if rc in (SHTB_ERR_BAD_ARG, SHTB_ERR_ALIGN, SHTB_ERR_WORKSPACE):
        raise ArgumentError(msg)
    raise BackendUnavailableError(operation, f"{msg} (status {rc})")


def profile_enable(on: bool) -> None:
    load().shtb_profile_enable(1 if on else 0)


def profile_read(max_kinds: int = 32) -> dict:
    """{kernel name: (total ms, launches)} of the launches recorded since profile_enable(True)."""
    import numpy as np

    names = ctypes.create_string_buffer(64 * max_kinds)
    tot = np.zeros(max_kinds, dtype=np.float64)
    cnt = np.zeros(max_kinds, dtype=np.int32)
    n = load().shtb_profile_read(max_kinds, names, tot.ctypes.data, cnt.ctypes.data)
    if n < 0:
        check(n, "profile_read")
    out = {}
    for i in range(min(n, max_kinds)):
        nm = names.raw[64 * i: 64 * i + 64].split(b"\0", 1)[0].decode()
        out[nm] = (float(tot[i]), int(cnt[i]))
    return out
