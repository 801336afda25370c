"""Host mirror of SHTnsKit's transform API on the B200 library.

Public names follow the reference (src/core_transforms.jl, src/sphtor_transforms.jl,
src/batch_transforms.jl, src/device_utils.jl): ``analysis``, ``synthesis``,
``analysis_sphtor``, ``synthesis_sphtor``, their ``_batch`` forms, in-place forms
(``analysis_into`` / ``synthesis_into`` for ``analysis!`` / ``synthesis!``),
``on_device``, ``to_device`` and ``gpu_clear_cache``.

Arrays use the reference's column-major layout. A grid is a tensor of shape
``(nlat, nlon[, nfields])`` whose memory is latitude-fastest (strides
``(1, nlat, nlat*nlon)``); coefficients are complex ``(lmax+1, mmax+1[, nfields])``
with l fastest. ``julia_empty`` allocates such tensors; inputs with other strides
are densified on the device first (``_gpu_adapter_dense``). Host (NumPy) inputs are
copied to the device (``_gpu_adapter_adapt``) and results stay on the device.

Every transform runs the CUDA library; there is no CPU path here. Autograd
(PyTorch's convention g = dL/dRe + i dL/dIm, the Zygote convention the
reference's rrules use) is provided by the library's adjoint kernels.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import ArgumentError, BackendUnavailableError, DimensionMismatch
from .config import SHTConfig

_PREC = {"fp64": _lib.SHTB_PREC_FP64, "mixed": _lib.SHTB_PREC_MIXED}


class CPU:
    """CPU device marker (src/devices.jl:7)."""

    def __repr__(self):
        return "CPU()"


class GPU:
    """GPU device marker (src/devices.jl:16)."""

    def __repr__(self):
        return "GPU()"


def on_device(x):
    """GPU() for CUDA tensors, CPU() otherwise (src/device_utils.jl:251-254)."""
    return GPU() if isinstance(x, torch.Tensor) and x.is_cuda else CPU()


# ---------------------------------------------------------------------------
# layout helpers
# ---------------------------------------------------------------------------

def julia_strides(shape) -> tuple:
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return tuple(st)


def julia_empty(shape, dtype, device) -> torch.Tensor:
    """Uninitialised tensor of ``shape`` with column-major (Julia) memory order."""
    shape = tuple(shape)
    rev = torch.empty(shape[::-1], dtype=dtype, device=device)
    return rev.permute(*reversed(range(len(shape))))


def is_julia_dense(t: torch.Tensor) -> bool:
    exp = julia_strides(t.shape)
    return all(t.shape[i] == 1 or t.stride(i) == exp[i] for i in range(t.dim()))


def _device_index(*vals) -> int:
    for v in vals:
        if isinstance(v, torch.Tensor) and v.is_cuda:
            return v.device.index
    if not torch.cuda.is_available():
        raise BackendUnavailableError("device", "no CUDA device is available")
    return torch.cuda.current_device()


def to_device(x, dtype, device_index: int) -> torch.Tensor:
    """Place ``x`` (NumPy array or tensor) on the device, column-major, with ``dtype``."""
    dev = torch.device("cuda", device_index)
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.asfortranarray(x))
    if not isinstance(x, torch.Tensor):
        raise ArgumentError(f"unsupported operand type {type(x)}")
    if x.device != dev or x.dtype != dtype or not is_julia_dense(x):
        out = julia_empty(x.shape, dtype, dev)
        out.copy_(x.to(dev) if x.dtype == dtype else x.to(dev).to(dtype))
        x = out
    return x


def to_host(t: torch.Tensor) -> np.ndarray:
    """Copy a column-major device tensor into a NumPy array indexed like the Julia array."""
    rev = t.permute(*reversed(range(t.dim()))).contiguous().cpu().numpy()
    return rev.T


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _stream(device_index: int) -> int:
    return torch.cuda.current_stream(device_index).cuda_stream


def _workspace(plan, op, nf, dtype_code, prec, device_index) -> tuple[torch.Tensor, int]:
    nb = plan.workspace_bytes(op, nf, dtype_code, prec)
    ws = torch.empty(max(nb, 256), dtype=torch.uint8, device=torch.device("cuda", device_index))
    return ws, nb


# ---------------------------------------------------------------------------
# raw device calls (column-major tensors, batched with a trailing field index)
# ---------------------------------------------------------------------------

def _prec_code(precision: str) -> int:
    try:
        return _PREC[precision]
    except KeyError:
        raise ArgumentError(f"precision must be 'fp64' or 'mixed', got {precision!r}") from None


def _types(prec: int):
    if prec == _lib.SHTB_PREC_FP64:
        return torch.float64, torch.complex128, _lib.SHTB_F64
    return torch.float32, torch.complex64, _lib.SHTB_F32


def _lcap(cfg: SHTConfig, lcap) -> int:
    if lcap is None:
        return cfg.lmax
    if not (0 <= lcap <= cfg.lmax):
        raise ArgumentError(f"lcap must satisfy 0 ≤ lcap ≤ lmax={cfg.lmax}")
    return int(lcap)


def synthesis_device(cfg: SHTConfig, alm: torch.Tensor, f_out: torch.Tensor, ltr: int, prec: int) -> torch.Tensor:
    dev = alm.device.index
    plan = cfg.plan(dev)
    nf = alm.shape[2]
    _, _, dcode = _types(prec)
    ws, nb = _workspace(plan, _lib.SHTB_OP_SYNTHESIS, nf, dcode, prec, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_synthesis(plan.handle, _ptr(alm), _ptr(f_out), nf, ltr, dcode, prec, _ptr(ws), nb,
                                        _stream(dev))
    _lib.check(rc, "synthesis")
    return f_out


def analysis_device(cfg: SHTConfig, f: torch.Tensor, alm_out: torch.Tensor, ltr: int, prec: int) -> torch.Tensor:
    dev = f.device.index
    plan = cfg.plan(dev)
    nf = f.shape[2]
    _, _, dcode = _types(prec)
    ws, nb = _workspace(plan, _lib.SHTB_OP_ANALYSIS, nf, dcode, prec, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_analysis(plan.handle, _ptr(f), _ptr(alm_out), nf, ltr, dcode, prec, _ptr(ws), nb,
                                       _stream(dev))
    _lib.check(rc, "analysis")
    return alm_out


def synthesis_sphtor_device(cfg, S, T, Vt, Vp, ltr: int):
    dev = S.device.index
    plan = cfg.plan(dev)
    nf = S.shape[2]
    ws, nb = _workspace(plan, _lib.SHTB_OP_SYNTHESIS_SPHTOR, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_synthesis_sphtor(plan.handle, _ptr(S), _ptr(T), _ptr(Vt), _ptr(Vp), nf, ltr,
                                               _lib.SHTB_F64, _lib.SHTB_PREC_FP64, _ptr(ws), nb, _stream(dev))
    _lib.check(rc, "synthesis_sphtor")
    return Vt, Vp


def analysis_sphtor_device(cfg, Vt, Vp, S, T, ltr: int):
    dev = Vt.device.index
    plan = cfg.plan(dev)
    nf = Vt.shape[2]
    ws, nb = _workspace(plan, _lib.SHTB_OP_ANALYSIS_SPHTOR, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_analysis_sphtor(plan.handle, _ptr(Vt), _ptr(Vp), _ptr(S), _ptr(T), nf, ltr,
                                              _lib.SHTB_F64, _lib.SHTB_PREC_FP64, _ptr(ws), nb, _stream(dev))
    _lib.check(rc, "analysis_sphtor")
    return S, T


def _adjoint_call(name, op, cfg, ins, outs, nf):
    dev = ins[0].device.index
    plan = cfg.plan(dev)
    ws, nb = _workspace(plan, op, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, dev)
    fn = getattr(_lib.load(), name)
    with torch.cuda.device(dev):
        rc = fn(plan.handle, *[_ptr(t) for t in ins], *[_ptr(t) for t in outs], nf, _ptr(ws), nb, _stream(dev))
    _lib.check(rc, name)


def adjoint_synthesis_device(cfg, ybar):
    nf = ybar.shape[2]
    abar = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, ybar.device)
    _adjoint_call("shtb_synthesis_adjoint", _lib.SHTB_OP_ANALYSIS, cfg, [ybar], [abar], nf)
    return abar


def adjoint_analysis_device(cfg, abar):
    nf = abar.shape[2]
    fbar = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, abar.device)
    _adjoint_call("shtb_analysis_adjoint", _lib.SHTB_OP_SYNTHESIS, cfg, [abar], [fbar], nf)
    return fbar


def adjoint_synthesis_sphtor_device(cfg, vtbar, vpbar):
    nf = vtbar.shape[2]
    S = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, vtbar.device)
    T = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, vtbar.device)
    _adjoint_call("shtb_synthesis_sphtor_adjoint", _lib.SHTB_OP_ANALYSIS_SPHTOR, cfg, [vtbar, vpbar], [S, T], nf)
    return S, T


def adjoint_analysis_sphtor_device(cfg, sbar, tbar):
    nf = sbar.shape[2]
    vt = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, sbar.device)
    vp = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, sbar.device)
    _adjoint_call("shtb_analysis_sphtor_adjoint", _lib.SHTB_OP_SYNTHESIS_SPHTOR, cfg, [sbar, tbar], [vt, vp], nf)
    return vt, vp


# ---------------------------------------------------------------------------
# autograd (the rrules of ext/SHTnsKitAdvancedADExt.jl:55-135, :198-246)
# ---------------------------------------------------------------------------

def _truncate_coeff_grad(cfg, g, ltr):
    if ltr < cfg.lmax:
        g = g.clone()
        g[ltr + 1:, :, :] = 0
        g[:, ltr + 1:, :] = 0
    return g


class _Synthesis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alm, cfg, ltr):
        ctx.cfg, ctx.ltr = cfg, ltr
        f = julia_empty((cfg.nlat, cfg.nlon, alm.shape[2]), torch.float64, alm.device)
        return synthesis_device(cfg, alm.detach(), f, ltr, _lib.SHTB_PREC_FP64)

    @staticmethod
    def backward(ctx, gf):
        cfg = ctx.cfg
        g = adjoint_synthesis_device(cfg, to_device(gf, torch.float64, gf.device.index))
        return _truncate_coeff_grad(cfg, g, ctx.ltr), None, None


class _Analysis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, cfg, ltr):
        ctx.cfg, ctx.ltr = cfg, ltr
        alm = julia_empty((cfg.lmax + 1, cfg.mmax + 1, f.shape[2]), torch.complex128, f.device)
        return analysis_device(cfg, f.detach(), alm, ltr, _lib.SHTB_PREC_FP64)

    @staticmethod
    def backward(ctx, ga):
        cfg = ctx.cfg
        ga = _truncate_coeff_grad(cfg, to_device(ga, torch.complex128, ga.device.index), ctx.ltr)
        return adjoint_analysis_device(cfg, to_device(ga, torch.complex128, ga.device.index)), None, None


class _SynthesisSphtor(torch.autograd.Function):
    @staticmethod
    def forward(ctx, S, T, cfg, ltr):
        ctx.cfg, ctx.ltr = cfg, ltr
        nf = S.shape[2]
        vt = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, S.device)
        vp = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, S.device)
        return synthesis_sphtor_device(cfg, S.detach(), T.detach(), vt, vp, ltr)

    @staticmethod
    def backward(ctx, gvt, gvp):
        cfg = ctx.cfg
        dev = (gvt if gvt is not None else gvp).device
        shape = (cfg.nlat, cfg.nlon, (gvt if gvt is not None else gvp).shape[2])
        gvt = torch.zeros(shape, dtype=torch.float64, device=dev) if gvt is None else gvt
        gvp = torch.zeros(shape, dtype=torch.float64, device=dev) if gvp is None else gvp
        S, T = adjoint_synthesis_sphtor_device(cfg, to_device(gvt, torch.float64, dev.index),
                                               to_device(gvp, torch.float64, dev.index))
        return _truncate_coeff_grad(cfg, S, ctx.ltr), _truncate_coeff_grad(cfg, T, ctx.ltr), None, None


class _AnalysisSphtor(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vt, vp, cfg, ltr):
        ctx.cfg, ctx.ltr = cfg, ltr
        nf = vt.shape[2]
        S = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, vt.device)
        T = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, vt.device)
        return analysis_sphtor_device(cfg, vt.detach(), vp.detach(), S, T, ltr)

    @staticmethod
    def backward(ctx, gs, gt):
        cfg = ctx.cfg
        ref = gs if gs is not None else gt
        shape = (cfg.lmax + 1, cfg.mmax + 1, ref.shape[2])
        gs = torch.zeros(shape, dtype=torch.complex128, device=ref.device) if gs is None else gs
        gt = torch.zeros(shape, dtype=torch.complex128, device=ref.device) if gt is None else gt
        gs = _truncate_coeff_grad(cfg, to_device(gs, torch.complex128, ref.device.index), ctx.ltr)
        gt = _truncate_coeff_grad(cfg, to_device(gt, torch.complex128, ref.device.index), ctx.ltr)
        vt, vp = adjoint_analysis_sphtor_device(cfg, gs, gt)
        return vt, vp, None, None


# ---------------------------------------------------------------------------
# public API
# ---------------------------------------------------------------------------

def _check_coeff_shape(cfg, a, batched):
    if a.dim() != (3 if batched else 2):
        raise DimensionMismatch(f"coefficients must be {'3' if batched else '2'}-dimensional, got {tuple(a.shape)}")
    if a.shape[0] != cfg.lmax + 1:
        raise DimensionMismatch(f"first dim must be lmax+1={cfg.lmax + 1}")
    if a.shape[1] != cfg.mmax + 1:
        raise DimensionMismatch(f"second dim must be mmax+1={cfg.mmax + 1}")


def _check_grid_shape(cfg, f, batched):
    if f.dim() != (3 if batched else 2):
        raise DimensionMismatch(f"field must be {'3' if batched else '2'}-dimensional, got {tuple(f.shape)}")
    if f.shape[0] != cfg.nlat:
        raise DimensionMismatch(f"first dim must be nlat={cfg.nlat}")
    if f.shape[1] != cfg.nlon:
        raise DimensionMismatch(f"second dim must be nlon={cfg.nlon}")


def _as_tensor(x):
    if isinstance(x, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(x))
    if isinstance(x, torch.Tensor):
        return x
    raise ArgumentError(f"unsupported operand type {type(x)}")


def _check_scratch(fft_scratch):
    if fft_scratch is not None:
        raise ArgumentError("CUDA scalar transforms do not accept a host fft_scratch")


def _cplx_call(name, op, cfg, src, dst, ltr):
    dev = src.device.index
    plan = cfg.plan(dev)
    nf = src.shape[2]
    ws, nb = _workspace(plan, op, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, dev)
    with torch.cuda.device(dev):
        rc = getattr(_lib.load(), name)(plan.handle, _ptr(src), _ptr(dst), nf, ltr, _ptr(ws), nb, _stream(dev))
    _lib.check(rc, name)
    return dst


def _synthesis_cplx(cfg, alm, batched, lcap, precision, out):
    # real_output = false: complex grid from the bins m >= 0 without the Hermitian fill
    # (src/core_transforms.jl:293-344), FP64 path
    if _prec_code(precision) != _lib.SHTB_PREC_FP64:
        raise BackendUnavailableError("synthesis", "complex output runs on the FP64 path only")
    a = _as_tensor(alm)
    _check_coeff_shape(cfg, a, batched)
    ltr = _lcap(cfg, lcap)
    dev = _device_index(alm, out)
    a3 = to_device(a if a.is_complex() else a.to(torch.complex128), torch.complex128, dev)
    a3 = a3 if batched else a3.unsqueeze(2)
    f = julia_empty((cfg.nlat, cfg.nlon, a3.shape[2]), torch.complex128, a3.device)
    _cplx_call("shtb_synthesis_cplx", _lib.SHTB_OP_SYNTHESIS, cfg, a3.detach(), f, ltr)
    if out is not None:
        out.copy_(f.reshape(out.shape))
        return out
    return f if batched else f[:, :, 0]


def _synthesis_impl(cfg, alm, batched, real_output, use_rfft, fft_scratch, lcap, precision, out=None):
    _check_scratch(fft_scratch)
    if use_rfft and not real_output:
        raise ArgumentError("use_rfft=true implies real_output")
    if use_rfft and cfg.mmax > cfg.nlon // 2:
        raise ArgumentError(f"use_rfft=true requires mmax ≤ nlon÷2, got mmax={cfg.mmax}, nlon={cfg.nlon}")
    if not real_output:
        return _synthesis_cplx(cfg, alm, batched, lcap, precision, out)
    a = _as_tensor(alm)
    _check_coeff_shape(cfg, a, batched)
    ltr = _lcap(cfg, lcap)
    prec = _prec_code(precision)
    rt, ct, _ = _types(prec)
    dev = _device_index(alm, out)
    a = to_device(a if a.is_complex() else a.to(ct), ct, dev)
    a3 = a if batched else a.unsqueeze(2)
    nf = a3.shape[2]
    if prec == _lib.SHTB_PREC_FP64 and a3.requires_grad and torch.is_grad_enabled() and out is None:
        f = _Synthesis.apply(a3, cfg, ltr)
    else:
        f = out if out is not None else julia_empty((cfg.nlat, cfg.nlon, nf), rt, a3.device)
        if out is not None and (out.dtype != rt or not is_julia_dense(out) or out.device != a3.device):
            tmp = julia_empty((cfg.nlat, cfg.nlon, nf), rt, a3.device)
            synthesis_device(cfg, a3.detach(), tmp, ltr, prec)
            out.copy_(tmp.reshape(out.shape))
            return out
        if out is not None:
            synthesis_device(cfg, a3.detach(), out.reshape(cfg.nlat, cfg.nlon, nf), ltr, prec)
            return out
        synthesis_device(cfg, a3.detach(), f, ltr, prec)
    return f if batched else f[:, :, 0]


def _analysis_impl(cfg, f, batched, use_rfft, fft_scratch, lcap, precision, out=None):
    _check_scratch(fft_scratch)
    t = _as_tensor(f)
    if t.is_complex():
        if use_rfft:
            raise ArgumentError("use_rfft=true requires a real-valued input")
        # complex field: coefficients from its bins m >= 0 (src/core_transforms.jl:169-207), FP64 path
        if _prec_code(precision) != _lib.SHTB_PREC_FP64:
            raise BackendUnavailableError("analysis", "complex fields run on the FP64 path only")
        _check_grid_shape(cfg, t, batched)
        ltr = _lcap(cfg, lcap)
        t3 = to_device(t, torch.complex128, _device_index(f, out))
        t3 = t3 if batched else t3.unsqueeze(2)
        a = julia_empty((cfg.lmax + 1, cfg.mmax + 1, t3.shape[2]), torch.complex128, t3.device)
        _cplx_call("shtb_analysis_cplx", _lib.SHTB_OP_ANALYSIS, cfg, t3.detach(), a, ltr)
        if out is not None:
            out.copy_(a.reshape(out.shape))
            return out
        return a if batched else a[:, :, 0]
    _check_grid_shape(cfg, t, batched)
    ltr = _lcap(cfg, lcap)
    prec = _prec_code(precision)
    rt, ct, _ = _types(prec)
    dev = _device_index(f, out)
    t = to_device(t, rt, dev)
    t3 = t if batched else t.unsqueeze(2)
    nf = t3.shape[2]
    if prec == _lib.SHTB_PREC_FP64 and t3.requires_grad and torch.is_grad_enabled() and out is None:
        a = _Analysis.apply(t3, cfg, ltr)
    else:
        a = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), ct, t3.device)
        analysis_device(cfg, t3.detach(), a, ltr, prec)
        if out is not None:
            out.copy_(a.reshape(out.shape))
            return out
    return a if batched else a[:, :, 0]


def synthesis(cfg: SHTConfig, alm, *, real_output: bool = True, use_rfft: bool = False, fft_scratch=None,
              lcap: int | None = None, precision: str = "fp64"):
    """Inverse scalar transform ``(lmax+1, mmax+1) -> (nlat, nlon)`` (src/core_transforms.jl:271-280)."""
    return _synthesis_impl(cfg, alm, False, real_output, use_rfft, fft_scratch, lcap, precision)


def analysis(cfg: SHTConfig, f, *, use_rfft: bool = False, fft_scratch=None, lcap: int | None = None,
             precision: str = "fp64"):
    """Forward scalar transform ``(nlat, nlon) -> (lmax+1, mmax+1)`` (src/core_transforms.jl:169-207)."""
    return _analysis_impl(cfg, f, False, use_rfft, fft_scratch, lcap, precision)


def synthesis_batch(cfg: SHTConfig, alm, *, real_output: bool = True, use_rfft: bool = False,
                    lcap: int | None = None, precision: str = "fp64"):
    """Batched synthesis ``(lmax+1, mmax+1, nf) -> (nlat, nlon, nf)`` (src/batch_transforms.jl:455-607)."""
    return _synthesis_impl(cfg, alm, True, real_output, use_rfft, None, lcap, precision)


def analysis_batch(cfg: SHTConfig, f, *, use_rfft: bool = False, lcap: int | None = None, precision: str = "fp64"):
    """Batched analysis ``(nlat, nlon, nf) -> (lmax+1, mmax+1, nf)`` (src/batch_transforms.jl:312-370)."""
    return _analysis_impl(cfg, f, True, use_rfft, None, lcap, precision)


def synthesis_into(cfg: SHTConfig, f_out: torch.Tensor, alm, *, real_output: bool = True, use_rfft: bool = False,
                   fft_scratch=None, lcap: int | None = None, precision: str = "fp64"):
    """In-place synthesis into ``f_out`` (``synthesis!``, src/core_transforms.jl:375-434)."""
    _check_grid_shape(cfg, f_out, f_out.dim() == 3)
    return _synthesis_impl(cfg, alm, f_out.dim() == 3, real_output, use_rfft, fft_scratch, lcap, precision, out=f_out)


def analysis_into(cfg: SHTConfig, alm_out: torch.Tensor, f, *, use_rfft: bool = False, fft_scratch=None,
                  lcap: int | None = None, precision: str = "fp64"):
    """In-place analysis into ``alm_out`` (``analysis!``, src/core_transforms.jl:215-263)."""
    _check_coeff_shape(cfg, alm_out, alm_out.dim() == 3)
    return _analysis_impl(cfg, f, alm_out.dim() == 3, use_rfft, fft_scratch, lcap, precision, out=alm_out)


def _sphtor_synth(cfg, S, T, batched, real_output, use_rfft, lcap):
    if use_rfft and not real_output:
        raise ArgumentError("use_rfft=true implies real_output")
    if not real_output:
        raise BackendUnavailableError("synthesis_sphtor", "complex output (real_output=false) is not implemented by this backend")
    s, t = _as_tensor(S), _as_tensor(T)
    for a, nm in ((s, "Slm"), (t, "Tlm")):
        if a.dim() != (3 if batched else 2) or a.shape[0] != cfg.lmax + 1 or a.shape[1] != cfg.mmax + 1:
            raise DimensionMismatch(f"{nm} dims")
    ltr = _lcap(cfg, lcap)
    dev = _device_index(S, T)
    s = to_device(s if s.is_complex() else s.to(torch.complex128), torch.complex128, dev)
    t = to_device(t if t.is_complex() else t.to(torch.complex128), torch.complex128, dev)
    s3 = s if batched else s.unsqueeze(2)
    t3 = t if batched else t.unsqueeze(2)
    if (s3.requires_grad or t3.requires_grad) and torch.is_grad_enabled():
        vt, vp = _SynthesisSphtor.apply(s3, t3, cfg, ltr)
    else:
        nf = s3.shape[2]
        vt = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, s3.device)
        vp = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, s3.device)
        synthesis_sphtor_device(cfg, s3.detach(), t3.detach(), vt, vp, ltr)
    return (vt, vp) if batched else (vt[:, :, 0], vp[:, :, 0])


def _sphtor_anal(cfg, Vt, Vp, batched, use_rfft, lcap):
    a, b = _as_tensor(Vt), _as_tensor(Vp)
    if a.is_complex() or b.is_complex():
        if use_rfft:
            raise ArgumentError("use_rfft=true requires real-valued Vt, Vp")
        raise BackendUnavailableError("analysis_sphtor", "complex-valued fields are not implemented by this backend")
    for v, nm in ((a, "Vt"), (b, "Vp")):
        if v.dim() != (3 if batched else 2) or v.shape[0] != cfg.nlat or v.shape[1] != cfg.nlon:
            raise DimensionMismatch(f"{nm} dims")
    ltr = _lcap(cfg, lcap)
    dev = _device_index(Vt, Vp)
    a = to_device(a, torch.float64, dev)
    b = to_device(b, torch.float64, dev)
    a3 = a if batched else a.unsqueeze(2)
    b3 = b if batched else b.unsqueeze(2)
    if (a3.requires_grad or b3.requires_grad) and torch.is_grad_enabled():
        S, T = _AnalysisSphtor.apply(a3, b3, cfg, ltr)
    else:
        nf = a3.shape[2]
        S = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, a3.device)
        T = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, a3.device)
        analysis_sphtor_device(cfg, a3.detach(), b3.detach(), S, T, ltr)
    return (S, T) if batched else (S[:, :, 0], T[:, :, 0])


def synthesis_sphtor(cfg: SHTConfig, Slm, Tlm, *, real_output: bool = True, use_rfft: bool = False,
                     lcap: int | None = None):
    """Spheroidal/toroidal synthesis to ``(Vt, Vp)`` (src/sphtor_transforms.jl:162-241)."""
    return _sphtor_synth(cfg, Slm, Tlm, False, real_output, use_rfft, lcap)


def analysis_sphtor(cfg: SHTConfig, Vt, Vp, *, use_rfft: bool = False, lcap: int | None = None):
    """Spheroidal/toroidal analysis of ``(Vt, Vp)`` (src/sphtor_transforms.jl:252-289)."""
    return _sphtor_anal(cfg, Vt, Vp, False, use_rfft, lcap)


def synthesis_sphtor_batch(cfg: SHTConfig, Slm, Tlm, *, real_output: bool = True, use_rfft: bool = False,
                           lcap: int | None = None):
    return _sphtor_synth(cfg, Slm, Tlm, True, real_output, use_rfft, lcap)


def analysis_sphtor_batch(cfg: SHTConfig, Vt, Vp, *, use_rfft: bool = False, lcap: int | None = None):
    return _sphtor_anal(cfg, Vt, Vp, True, use_rfft, lcap)


# ---------------------------------------------------------------------------
# packed LM layout (SHTns order: m blocks of l = m..lmax, src/layout.jl:88-339)
# ---------------------------------------------------------------------------

def nlm_calc(lmax: int, mmax: int, mres: int) -> int:
    """Number of packed coefficients (src/layout.jl:88-101)."""
    if lmax < 0 or mmax < 0 or mres < 1:
        raise ArgumentError("invalid sizes")
    if mmax > lmax:
        return 0
    return sum(lmax - m + 1 for m in range(0, mmax + 1, mres))


def LM_index(lmax: int, mres: int, l: int, m: int) -> int:
    """0-based packed index of (l, m) (src/layout.jl:143-162)."""
    if m < 0:
        raise ArgumentError("m must be ≥ 0 for packed layout")
    if m % mres:
        raise ArgumentError("m must be a multiple of mres")
    if not (m <= l <= lmax):
        raise ArgumentError("require m ≤ l ≤ lmax")
    im = m // mres
    return ((im * (2 * lmax + 2 - (im + 1) * mres)) >> 1) + l


def _lm_gather_index(cfg: SHTConfig, device) -> torch.Tensor:
    """Dense column-major offsets l + (lmax+1) m of the packed entries, in packed order."""
    idx = [l + (cfg.lmax + 1) * m for m in range(0, cfg.mmax + 1, cfg.mres) for l in range(m, cfg.lmax + 1)]
    return torch.tensor(idx, dtype=torch.long, device=device)


def pack_lm(cfg: SHTConfig, A):
    """Dense (lmax+1, mmax+1) coefficients to the packed LM vector (src/layout.jl:315-339);
    orders off the mres lattice are skipped."""
    a = _as_tensor(A)
    _check_coeff_shape(cfg, a, False)
    dev = _device_index(A)
    a = to_device(a if a.is_complex() else a.to(torch.complex128), a.dtype if a.is_complex() else torch.complex128, dev)
    flat = a.permute(1, 0).reshape(-1)                    # column-major memory order
    return flat[_lm_gather_index(cfg, a.device)].contiguous()


def unpack_lm(cfg: SHTConfig, Qlm):
    """Packed LM vector to dense (lmax+1, mmax+1) coefficients, zero where the packed layout
    has no entry (src/layout.jl:282-307)."""
    q = _as_tensor(Qlm)
    if q.dim() != 1 or q.shape[0] != cfg.nlm:
        raise DimensionMismatch(f"Qlm must have length {cfg.nlm}")
    dev = _device_index(Qlm)
    q = q.to(torch.device("cuda", dev))
    if not q.is_complex():
        q = q.to(torch.complex128)
    out = julia_empty((cfg.lmax + 1, cfg.mmax + 1), q.dtype, q.device)
    out.zero_()
    out.permute(1, 0).reshape(-1)[_lm_gather_index(cfg, q.device)] = q
    return out


def _packed_synth(cfg, Qlm, batched, lcap, precision):
    q = _as_tensor(Qlm)
    if q.dim() != (2 if batched else 1) or q.shape[0] != cfg.nlm:
        raise DimensionMismatch(f"Qlm must have length {cfg.nlm}")
    ltr = _lcap(cfg, lcap)
    prec = _prec_code(precision)
    rt, ct, dcode = _types(prec)
    dev = _device_index(Qlm)
    q = to_device(q if q.is_complex() else q.to(ct), ct, dev)
    q2 = q if batched else q.unsqueeze(1)
    nf = q2.shape[1]
    f = julia_empty((cfg.nlat, cfg.nlon, nf), rt, q2.device)
    plan = cfg.plan(dev)
    ws, nb = _workspace(plan, _lib.SHTB_OP_SYNTHESIS, nf, dcode, prec, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_synthesis_packed(plan.handle, _ptr(q2), _ptr(f), nf, ltr, dcode, prec, _ptr(ws), nb,
                                               _stream(dev))
    _lib.check(rc, "synthesis_packed")
    flat = f.permute(2, 1, 0).reshape(nf, cfg.nlat * cfg.nlon).permute(1, 0)   # vec(f) per field
    return flat if batched else flat[:, 0]


def _packed_anal(cfg, Vr, batched, lcap, precision):
    v = _as_tensor(Vr)
    if v.is_complex() or v.dim() != (2 if batched else 1) or v.shape[0] != cfg.nlat * cfg.nlon:
        raise DimensionMismatch(f"Vr must have length {cfg.nlat * cfg.nlon}")
    ltr = _lcap(cfg, lcap)
    prec = _prec_code(precision)
    rt, ct, dcode = _types(prec)
    dev = _device_index(Vr)
    v = to_device(v, rt, dev)
    v2 = v if batched else v.unsqueeze(1)
    nf = v2.shape[1]
    grid = v2.permute(1, 0).reshape(nf, cfg.nlon, cfg.nlat).permute(2, 1, 0)   # (nlat, nlon, nf), column-major
    if not is_julia_dense(grid):
        g = julia_empty((cfg.nlat, cfg.nlon, nf), rt, v2.device)
        g.copy_(grid)
        grid = g
    q = julia_empty((cfg.nlm, nf), ct, v2.device)
    plan = cfg.plan(dev)
    ws, nb = _workspace(plan, _lib.SHTB_OP_ANALYSIS, nf, dcode, prec, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_analysis_packed(plan.handle, _ptr(grid), _ptr(q), nf, ltr, dcode, prec, _ptr(ws), nb,
                                              _stream(dev))
    _lib.check(rc, "analysis_packed")
    return q if batched else q[:, 0]


def synthesis_packed(cfg: SHTConfig, Qlm, *, precision: str = "fp64"):
    """Packed LM coefficients (length nlm) to the flattened real grid vec(f), length nlat·nlon
    (src/transforms.jl:144-155)."""
    return _packed_synth(cfg, Qlm, False, None, precision)


def synthesis_packed_l(cfg: SHTConfig, Qlm, ltr: int, *, precision: str = "fp64"):
    """``synthesis_packed`` using degrees l ≤ ltr only (src/transforms.jl:209-227)."""
    return _packed_synth(cfg, Qlm, False, ltr, precision)


def analysis_packed(cfg: SHTConfig, Vr, *, precision: str = "fp64"):
    """Flattened real grid (length nlat·nlon) to packed LM coefficients (src/transforms.jl:125-136)."""
    return _packed_anal(cfg, Vr, False, None, precision)


def analysis_packed_l(cfg: SHTConfig, Vr, ltr: int, *, precision: str = "fp64"):
    """``analysis_packed`` truncated to l ≤ ltr; the other packed entries are zero
    (src/transforms.jl:183-203)."""
    return _packed_anal(cfg, Vr, False, ltr, precision)


def synthesis_packed_batch(cfg: SHTConfig, Qlm, *, lcap: int | None = None, precision: str = "fp64"):
    """Fields along the trailing axis: (nlm, nfields) -> (nlat·nlon, nfields)."""
    return _packed_synth(cfg, Qlm, True, lcap, precision)


def analysis_packed_batch(cfg: SHTConfig, Vr, *, lcap: int | None = None, precision: str = "fp64"):
    """(nlat·nlon, nfields) -> (nlm, nfields)."""
    return _packed_anal(cfg, Vr, True, lcap, precision)


# ---------------------------------------------------------------------------
# diagonal spectral operators and divergence/vorticity spectra
# ---------------------------------------------------------------------------

def _spectral_op(name, op, cfg, src, out):
    a = _as_tensor(src)
    if not a.is_complex():
        a = a.to(torch.complex128)
    if a.dim() not in (2, 3) or a.shape[0] != cfg.lmax + 1 or a.shape[1] != cfg.mmax + 1:
        raise DimensionMismatch("spectral input dims")
    if a.dtype not in (torch.complex64, torch.complex128):
        raise ArgumentError(f"{name}: complex64 or complex128 coefficients expected")
    dev = _device_index(src) if out is None else _device_index(src, out)
    a = to_device(a, a.dtype, dev)
    if out is None:
        o = julia_empty(tuple(a.shape), a.dtype, a.device)
    else:
        o = out
        if not isinstance(o, torch.Tensor) or not o.is_cuda or tuple(o.shape) != tuple(a.shape):
            raise DimensionMismatch(f"{name}: output dims")
        if o.dtype != a.dtype or not is_julia_dense(o):
            raise ArgumentError(f"{name}: output must be a column-major {a.dtype} device array")
    nf = a.shape[2] if a.dim() == 3 else 1
    plan = cfg.plan(dev)
    dcode = _lib.SHTB_F64 if a.dtype == torch.complex128 else _lib.SHTB_F32
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_spectral_op(plan.handle, op, _ptr(a), _ptr(o), nf, dcode, _stream(dev))
    _lib.check(rc, name)
    return o


def divergence_from_spheroidal(cfg: SHTConfig, Slm):
    """δ_lm = −l(l+1) S_lm, zero for l < max(1, m) and m off the mres lattice
    (src/sphtor_transforms.jl:744-783). Coefficients (lmax+1, mmax+1[, nfields])."""
    return _spectral_op("divergence_from_spheroidal", _lib.SHTB_SPEC_NEG_LL, cfg, Slm, None)


def divergence_from_spheroidal_into(cfg: SHTConfig, out, Slm):
    """``divergence_from_spheroidal!``: writes into ``out``, which may be ``Slm`` itself."""
    return _spectral_op("divergence_from_spheroidal!", _lib.SHTB_SPEC_NEG_LL, cfg, Slm, out)


def spheroidal_from_divergence(cfg: SHTConfig, dlm):
    """S_lm = −δ_lm / (l(l+1)) for l ≥ max(1, m), else zero (src/sphtor_transforms.jl:790-831)."""
    return _spectral_op("spheroidal_from_divergence", _lib.SHTB_SPEC_INV_NEG_LL, cfg, dlm, None)


def spheroidal_from_divergence_into(cfg: SHTConfig, out, dlm):
    """``spheroidal_from_divergence!``: writes into ``out``, which may be ``dlm`` itself."""
    return _spectral_op("spheroidal_from_divergence!", _lib.SHTB_SPEC_INV_NEG_LL, cfg, dlm, out)


def vorticity_from_toroidal(cfg: SHTConfig, Tlm):
    """ζ_lm = −l(l+1) T_lm (src/sphtor_transforms.jl:838-877)."""
    return _spectral_op("vorticity_from_toroidal", _lib.SHTB_SPEC_NEG_LL, cfg, Tlm, None)


def vorticity_from_toroidal_into(cfg: SHTConfig, out, Tlm):
    """``vorticity_from_toroidal!``: writes into ``out``, which may be ``Tlm`` itself."""
    return _spectral_op("vorticity_from_toroidal!", _lib.SHTB_SPEC_NEG_LL, cfg, Tlm, out)


def toroidal_from_vorticity(cfg: SHTConfig, zlm):
    """T_lm = −ζ_lm / (l(l+1)) (src/sphtor_transforms.jl:884-925)."""
    return _spectral_op("toroidal_from_vorticity", _lib.SHTB_SPEC_INV_NEG_LL, cfg, zlm, None)


def toroidal_from_vorticity_into(cfg: SHTConfig, out, zlm):
    """``toroidal_from_vorticity!``: writes into ``out``, which may be ``zlm`` itself."""
    return _spectral_op("toroidal_from_vorticity!", _lib.SHTB_SPEC_INV_NEG_LL, cfg, zlm, out)


def gpu_apply_laplacian(cfg: SHTConfig, coeffs):
    """``gpu_apply_laplacian!``: in place, a_lm ← −l(l+1) a_lm on a device array (zero for
    l < max(1, m) and m off the mres lattice; ext/GPUCommon.jl:1501-1512,
    ext/SHTnsKitGPUExt.jl:2382-2389). Returns ``coeffs``."""
    if not isinstance(coeffs, torch.Tensor) or not coeffs.is_cuda:
        raise ArgumentError("gpu_apply_laplacian!: coefficients must be a device array")
    return _spectral_op("gpu_apply_laplacian!", _lib.SHTB_SPEC_NEG_LL, cfg, coeffs, coeffs)


def _divvort_synth(cfg, D, Z, batched, lcap):
    d, z = _as_tensor(D), _as_tensor(Z)
    for a, nm in ((d, "div"), (z, "vort")):
        if a.dim() != (3 if batched else 2) or a.shape[0] != cfg.lmax + 1 or a.shape[1] != cfg.mmax + 1:
            raise DimensionMismatch(f"{nm} dims")
    ltr = _lcap(cfg, lcap)
    dev = _device_index(D, Z)
    d = to_device(d if d.is_complex() else d.to(torch.complex128), torch.complex128, dev)
    z = to_device(z if z.is_complex() else z.to(torch.complex128), torch.complex128, dev)
    d3 = d if batched else d.unsqueeze(2)
    z3 = z if batched else z.unsqueeze(2)
    nf = d3.shape[2]
    vt = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, d3.device)
    vp = julia_empty((cfg.nlat, cfg.nlon, nf), torch.float64, d3.device)
    plan = cfg.plan(dev)
    ws, nb = _workspace(plan, _lib.SHTB_OP_SYNTHESIS_SPHTOR, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_synthesis_divvort(plan.handle, _ptr(d3), _ptr(z3), _ptr(vt), _ptr(vp), nf, ltr,
                                                _lib.SHTB_F64, _lib.SHTB_PREC_FP64, _ptr(ws), nb, _stream(dev))
    _lib.check(rc, "synthesis_divvort")
    return (vt, vp) if batched else (vt[:, :, 0], vp[:, :, 0])


def _divvort_anal(cfg, Vt, Vp, batched, lcap):
    a, b = _as_tensor(Vt), _as_tensor(Vp)
    for v, nm in ((a, "Vt"), (b, "Vp")):
        if v.is_complex() or v.dim() != (3 if batched else 2) or v.shape[0] != cfg.nlat or v.shape[1] != cfg.nlon:
            raise DimensionMismatch(f"{nm} dims")
    ltr = _lcap(cfg, lcap)
    dev = _device_index(Vt, Vp)
    a3 = to_device(a, torch.float64, dev)
    b3 = to_device(b, torch.float64, dev)
    a3 = a3 if batched else a3.unsqueeze(2)
    b3 = b3 if batched else b3.unsqueeze(2)
    nf = a3.shape[2]
    D = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, a3.device)
    Z = julia_empty((cfg.lmax + 1, cfg.mmax + 1, nf), torch.complex128, a3.device)
    plan = cfg.plan(dev)
    ws, nb = _workspace(plan, _lib.SHTB_OP_ANALYSIS_SPHTOR, nf, _lib.SHTB_F64, _lib.SHTB_PREC_FP64, dev)
    with torch.cuda.device(dev):
        rc = _lib.load().shtb_analysis_divvort(plan.handle, _ptr(a3), _ptr(b3), _ptr(D), _ptr(Z), nf, ltr,
                                               _lib.SHTB_F64, _lib.SHTB_PREC_FP64, _ptr(ws), nb, _stream(dev))
    _lib.check(rc, "analysis_divvort")
    return (D, Z) if batched else (D[:, :, 0], Z[:, :, 0])


def synthesis_divvort(cfg: SHTConfig, div, vort, *, lcap: int | None = None):
    """``synthesis_sphtor(cfg, spheroidal_from_divergence(cfg, div), toroidal_from_vorticity(cfg, vort))``
    in one pass: the −1/(l(l+1)) factor is applied as the coefficients enter the Legendre stage."""
    return _divvort_synth(cfg, div, vort, False, lcap)


def analysis_divvort(cfg: SHTConfig, Vt, Vp, *, lcap: int | None = None):
    """``(divergence_from_spheroidal(S), vorticity_from_toroidal(T))`` of ``analysis_sphtor(cfg, Vt, Vp)``
    in one pass: the −l(l+1) factor is applied as the coefficients leave the Legendre stage."""
    return _divvort_anal(cfg, Vt, Vp, False, lcap)


def synthesis_divvort_batch(cfg: SHTConfig, div, vort, *, lcap: int | None = None):
    return _divvort_synth(cfg, div, vort, True, lcap)


def analysis_divvort_batch(cfg: SHTConfig, Vt, Vp, *, lcap: int | None = None):
    return _divvort_anal(cfg, Vt, Vp, True, lcap)


def synthesis_qst(cfg: SHTConfig, Qlm, Slm, Tlm, *, real_output: bool = True, use_rfft: bool = False,
                  lcap: int | None = None):
    """Radial/spheroidal/toroidal synthesis to ``(Vr, Vt, Vp)`` (src/qst_transforms.jl:112-135):
    the scalar synthesis of Q and the spheroidal/toroidal synthesis of (S, T) on one grid."""
    vr = synthesis(cfg, Qlm, real_output=real_output, use_rfft=use_rfft, lcap=lcap)
    vt, vp = synthesis_sphtor(cfg, Slm, Tlm, real_output=real_output, use_rfft=use_rfft, lcap=lcap)
    return vr, vt, vp


def analysis_qst(cfg: SHTConfig, Vr, Vt, Vp, *, use_rfft: bool = False, lcap: int | None = None):
    """``(Vr, Vt, Vp)`` to ``(Q, S, T)`` (src/qst_transforms.jl:138-160)."""
    q = analysis(cfg, Vr, use_rfft=use_rfft, lcap=lcap)
    s, t = analysis_sphtor(cfg, Vt, Vp, use_rfft=use_rfft, lcap=lcap)
    return q, s, t


def synthesis_qst_batch(cfg: SHTConfig, Qlm, Slm, Tlm, *, real_output: bool = True, use_rfft: bool = False,
                        lcap: int | None = None):
    """Batched QST synthesis (src/batch_transforms.jl:830-905)."""
    vr = synthesis_batch(cfg, Qlm, real_output=real_output, use_rfft=use_rfft, lcap=lcap)
    vt, vp = synthesis_sphtor_batch(cfg, Slm, Tlm, real_output=real_output, use_rfft=use_rfft, lcap=lcap)
    return vr, vt, vp


def analysis_qst_batch(cfg: SHTConfig, Vr, Vt, Vp, *, use_rfft: bool = False, lcap: int | None = None):
    """Batched QST analysis (src/batch_transforms.jl:905-985)."""
    q = analysis_batch(cfg, Vr, use_rfft=use_rfft, lcap=lcap)
    s, t = analysis_sphtor_batch(cfg, Vt, Vp, use_rfft=use_rfft, lcap=lcap)
    return q, s, t


def gpu_clear_cache(cfg: SHTConfig | None = None) -> None:
    """Release device plans (``gpu_clear_cache!``, src/device_utils.jl:296-301)."""
    if cfg is not None:
        cfg.clear_plans()
