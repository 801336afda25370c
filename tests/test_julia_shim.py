"""The Julia adapter (`julia/SHTnsKitB200/src/SHTnsKitB200.jl`) against the C ABI.

Julia is not installed here, so the shim is checked in two ways:

* CPU: every `ccall` in the shim is parsed and its argument-type tuple and return type
  are compared with the prototype in `include/shtb200.h` and with the ctypes signature of
  the Python mirror; the number of arguments passed must match the tuple.
* GPU: the exact argument tuples that the shim's batch, in-place, complex, vector and
  batch-adjoint methods pass (same workspace op codes, dtype/precision codes, lcap and
  nfields) are issued through ctypes and checked against the FP64 oracle.
"""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SHIM = ROOT / "shtnskit.jl_b200" / "julia" / "SHTnsKitB200" / "src" / "SHTnsKitB200.jl"
HEADER = ROOT / "include" / "shtb200.h"

JL_KIND = {"Cint": "int", "Csize_t": "size", "Cdouble": "double", "UInt64": "u64", "Cstring": "ptr"}


def jl_kind(t: str) -> str:
    t = t.strip()
    if t.startswith(("Ptr{", "CuPtr{", "Ref{")):
        return "ptr"
    return JL_KIND[t]


def c_kind(decl: str) -> str:
    decl = decl.strip()
    if "*" in decl:
        return "ptr"
    base = decl.rsplit(" ", 1)[0] if " " in decl else decl
    base = base.replace("const ", "").strip()
    return {"int": "int", "size_t": "size", "double": "double", "uint64_t": "u64"}[base]


def split_top(s: str) -> list[str]:
    """Split at commas that are not nested in (), {} or []."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [x.strip() for x in out if x.strip()]


def matching(s: str, i: int) -> int:
    """Index of the parenthesis closing the one at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    raise ValueError("unbalanced")


def header_prototypes() -> dict:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    protos = {}
    for m in re.finditer(r"(int|size_t|const char\s*\*)\s*(shtb_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.S):
        ret, name, params = m.group(1), m.group(2), m.group(3).strip()
        kinds = [] if params in ("", "void") else [c_kind(p) for p in split_top(params)]
        protos[name] = ({"int": "int", "size_t": "size"}.get(ret.strip(), "ptr"), kinds)
    return protos


def shim_ccalls() -> list:
    """(symbol or None for a dynamic one, return kind, arg kinds, number of args passed or None)."""
    src = SHIM.read_text()
    calls = []
    for m in re.finditer(r"ccall\(", src):
        open_i = m.end() - 1
        body = src[open_i + 1:matching(src, open_i)]
        parts = split_top(body)
        target, ret, tup = parts[0], parts[1], parts[2]
        sm = re.match(r"\(\s*:(\w+)\s*,\s*LIB\s*\)", target)
        sym = sm.group(1) if sm else None
        assert tup.startswith("(") and tup.endswith(")")
        kinds = [jl_kind(t) for t in split_top(tup[1:-1])]
        args = parts[3:]
        nargs = None if any(a.endswith("...") for a in args) else len(args)
        calls.append((sym, jl_kind(ret), kinds, nargs))
    return calls


def test_shim_ccalls_match_header_and_ctypes():
    from shtb200 import _lib

    protos = header_prototypes()
    calls = shim_ccalls()
    assert len(calls) >= 15
    py_kind = {ctypes.c_void_p: "ptr", ctypes.c_int: "int", ctypes.c_size_t: "size", ctypes.c_double: "double",
               ctypes.c_uint64: "u64", ctypes.c_char_p: "ptr"}
    static = [c for c in calls if c[0] is not None]
    for sym, ret, kinds, nargs in static:
        assert sym in protos, f"shim calls {sym}, which the header does not declare"
        cret, ckinds = protos[sym]
        assert ret == cret, f"{sym}: return type {ret} vs header {cret}"
        assert kinds == ckinds, f"{sym}: shim types {kinds} vs header {ckinds}"
        if nargs is not None:
            assert nargs == len(kinds), f"{sym}: {nargs} arguments passed for {len(kinds)} types"
        pret, pargs = _lib.SIGNATURES[sym]
        # ctypes.c_size_t is ctypes.c_uint64 on LP64, so both read as "u64" there
        pk = [py_kind.get(a, "ptr") for a in pargs]
        ck = ["u64" if k == "size" else k for k in ckinds]
        assert pk == ck, f"{sym}: ctypes mirror {pk} vs header {ckinds}"
    # the adjoint helper's two dynamic-symbol ccalls: one input/one output, two/two
    dyn = sorted((c for c in calls if c[0] is None), key=lambda c: len(c[2]))
    assert [len(c[2]) for c in dyn] == [7, 9]
    src = SHIM.read_text()
    adj = set(re.findall(r"_adjoint\(:(\w+)", src))
    assert adj == {"shtb_synthesis_adjoint", "shtb_analysis_adjoint", "shtb_synthesis_sphtor_adjoint",
                   "shtb_analysis_sphtor_adjoint"}
    for sym in adj:
        kinds = dyn[1][2] if "sphtor" in sym else dyn[0][2]
        assert kinds == protos[sym][1], f"{sym}: adjoint helper types {kinds} vs header {protos[sym][1]}"


def test_shim_defines_reference_methods():
    """The direct methods of the reference's CUDA extension exist in the shim, with the
    reference's positional signature (ext/SHTnsKitGPUExt.jl:1294-1315, :1845-2020)."""
    src = SHIM.read_text()
    wanted = [
        r"SHTnsKit\.analysis_batch\(::SHTnsKit\.GPU, cfg::SHTnsKit\.SHTConfig, f::CuArray\{<:Real,3\}",
        r"SHTnsKit\.analysis_batch!\(::SHTnsKit\.GPU, cfg::SHTnsKit\.SHTConfig, output::CuArray\{Complex\{T\},3\}",
        r"SHTnsKit\.synthesis_batch\(::SHTnsKit\.GPU, cfg::SHTnsKit\.SHTConfig, alm::CuArray\{<:Complex,3\}",
        r"SHTnsKit\.synthesis_batch!\(::SHTnsKit\.GPU, cfg::SHTnsKit\.SHTConfig, output::CuArray\{T,3\}",
        r"SHTnsKit\.synthesis_batch_cplx\(::SHTnsKit\.GPU",
        r"SHTnsKit\.analysis_sphtor_batch\(::SHTnsKit\.GPU, cfg::SHTnsKit\.SHTConfig, Vt::CuArray\{<:Real,3\}",
        r"SHTnsKit\.synthesis_sphtor_batch\(::SHTnsKit\.GPU, cfg::SHTnsKit\.SHTConfig, S::CuArray\{<:Complex,3\}",
        r"SHTnsKit\.synthesis!\(::SHTnsKit\.GPU, plan::SHTnsKit\.SHTPlan",
        r"SHTnsKit\.analysis!\(::SHTnsKit\.GPU, plan::SHTnsKit\.SHTPlan",
        r"SHTnsKit\.synthesis!\(cfg::SHTnsKit\.SHTConfig, output::CuArray",
        r"SHTnsKit\.analysis!\(cfg::SHTnsKit\.SHTConfig, output::CuArray",
        r"ChainRulesCore\.rrule\(::typeof\(SHTnsKit\.synthesis_batch\)",
        r"ChainRulesCore\.rrule\(::typeof\(SHTnsKit\.analysis_batch\)",
        r"function precision_of\(",
    ]
    for w in wanted:
        assert re.search(w, src), f"shim lacks {w}"


# ---------------------------------------------------------------------------------- GPU
# The shim's argument tuples, issued through ctypes with the same codes.

SYN, ANA, SYN_V, ANA_V = 0, 1, 2, 3
F64, F32, PREC_FP64, PREC_MIXED = 0, 1, 0, 1


def _gpu_env():
    import torch
    import shtb200 as sht
    from shtb200 import _lib
    from oracle import sht_oracle as so
    return torch, sht, _lib, so


def _ws(torch, lib, plan, op, nf, dt, prec):
    # workspace(p, op, nf, dtype, prec) = CuArray{UInt8}(undef, max(256, shtb_workspace_bytes(...)))
    n = max(256, lib.shtb_workspace_bytes(plan.handle, op, nf, dt, prec))
    return torch.empty(n, dtype=torch.uint8, device="cuda:0"), n


@pytest.mark.gpu
def test_shim_batch_and_inplace_tuples():
    torch, sht, _lib, so = _gpu_env()
    from _util import rand_alm, rel_l2
    lib = _lib.load()
    lmax, nlat, nlon, nf = 31, 32, 64, 3
    cfg = sht.create_gauss_config(lmax, nlat, nlon=nlon)
    oc = so.create_gauss_config(lmax, nlat, nlon=nlon)
    plan = cfg.plan(0)
    st = torch.cuda.current_stream(0).cuda_stream
    a = rand_alm(lmax, lmax, nf, seed=11)
    ref_f = so.synthesis_batch(oc, a)

    def run(sym, ins, outs, tail, op, dt, prec, nfc):
        ws, n = _ws(torch, lib, plan, op, nfc, dt, prec)
        fn = getattr(lib, sym)
        rc = fn(plan.handle, *[t.data_ptr() for t in ins], *[t.data_ptr() for t in outs], *tail, ws.data_ptr(), n, st)
        _lib.check(rc, sym)
        torch.cuda.synchronize()

    # synthesis_batch(::GPU, cfg, alm::CuArray{ComplexF64,3}) -> _synthesis!(f, cfg, alm, lmax, FP64)
    alm = sht.to_device(a, torch.complex128, 0)
    f = sht.julia_empty((nlat, nlon, nf), torch.float64, "cuda:0")
    run("shtb_synthesis", [alm], [f], (nf, lmax, F64, PREC_FP64), SYN, F64, PREC_FP64, nf)
    assert rel_l2(sht.to_host(f), ref_f) <= 1e-12

    # analysis_batch(::GPU, cfg, f::CuArray{Float64,3})
    out = sht.julia_empty((lmax + 1, lmax + 1, nf), torch.complex128, "cuda:0")
    run("shtb_analysis", [f], [out], (nf, lmax, F64, PREC_FP64), ANA, F64, PREC_FP64, nf)
    assert rel_l2(sht.to_host(out), so.analysis_batch(oc, ref_f)) <= 1e-12

    # Float32 arrays: the documented rule selects the mixed path (dtype F32, precision MIXED)
    alm32 = sht.to_device(a, torch.complex64, 0)
    f32 = sht.julia_empty((nlat, nlon, nf), torch.float32, "cuda:0")
    run("shtb_synthesis", [alm32], [f32], (nf, lmax, F32, PREC_MIXED), SYN, F32, PREC_MIXED, nf)
    assert rel_l2(sht.to_host(f32), ref_f) <= 1e-6

    # synthesis!(::GPU, plan, output::CuMatrix, alm::CuMatrix): nf = 1 into the caller's matrix,
    # a slice of a larger buffer, with lcap = lmax
    big = sht.julia_empty((nlat, nlon, 2), torch.float64, "cuda:0")
    big.fill_(7.0)
    one = big[:, :, 1:2]
    run("shtb_synthesis", [alm[:, :, 1:2]], [one], (1, lmax, F64, PREC_FP64), SYN, F64, PREC_FP64, 1)
    h = sht.to_host(big)
    assert np.all(h[:, :, 0] == 7.0)
    assert rel_l2(h[:, :, 1], ref_f[:, :, 1]) <= 1e-12

    # analysis!(::GPU, plan, output::CuMatrix, field::CuMatrix)
    o1 = sht.julia_empty((lmax + 1, lmax + 1, 1), torch.complex128, "cuda:0")
    run("shtb_analysis", [f[:, :, 2:3]], [o1], (1, lmax, F64, PREC_FP64), ANA, F64, PREC_FP64, 1)
    assert rel_l2(sht.to_host(o1)[:, :, 0], so.analysis(oc, ref_f[:, :, 2])) <= 1e-12

    # synthesis_batch(...; real_output=false) / synthesis_batch_cplx -> shtb_synthesis_cplx
    g = sht.julia_empty((nlat, nlon, nf), torch.complex128, "cuda:0")
    run("shtb_synthesis_cplx", [alm], [g], (nf, lmax), SYN, F64, PREC_FP64, nf)
    gref = so.synthesis_batch(oc, a, real_output=False)
    assert rel_l2(sht.to_host(g), gref) <= 1e-12
    # analysis_batch! of complex fields -> shtb_analysis_cplx
    oc2 = sht.julia_empty((lmax + 1, lmax + 1, nf), torch.complex128, "cuda:0")
    run("shtb_analysis_cplx", [g], [oc2], (nf, lmax), ANA, F64, PREC_FP64, nf)
    aref = np.stack([so.analysis(oc, gref[:, :, k]) for k in range(nf)], axis=2)
    assert rel_l2(sht.to_host(oc2), aref) <= 1e-12

    # synthesis_sphtor_batch / analysis_sphtor_batch
    S = rand_alm(lmax, lmax, nf, seed=12, lmin=1)
    T = rand_alm(lmax, lmax, nf, seed=13, lmin=1)
    Sd, Td = sht.to_device(S, torch.complex128, 0), sht.to_device(T, torch.complex128, 0)
    Vt = sht.julia_empty((nlat, nlon, nf), torch.float64, "cuda:0")
    Vp = sht.julia_empty((nlat, nlon, nf), torch.float64, "cuda:0")
    run("shtb_synthesis_sphtor", [Sd, Td], [Vt, Vp], (nf, lmax, F64, PREC_FP64), SYN_V, F64, PREC_FP64, nf)
    vt_ref, vp_ref = so.synthesis_sphtor_batch(oc, S, T)
    assert rel_l2(sht.to_host(Vt), vt_ref) <= 1e-12 and rel_l2(sht.to_host(Vp), vp_ref) <= 1e-12
    S2 = sht.julia_empty((lmax + 1, lmax + 1, nf), torch.complex128, "cuda:0")
    T2 = sht.julia_empty((lmax + 1, lmax + 1, nf), torch.complex128, "cuda:0")
    run("shtb_analysis_sphtor", [Vt, Vp], [S2, T2], (nf, lmax, F64, PREC_FP64), ANA_V, F64, PREC_FP64, nf)
    s_ref, t_ref = so.analysis_sphtor_batch(oc, vt_ref, vp_ref)
    assert rel_l2(sht.to_host(S2), s_ref) <= 1e-12 and rel_l2(sht.to_host(T2), t_ref) <= 1e-12


@pytest.mark.gpu
def test_shim_batch_rrule_tuples():
    """The batch rrules' pullbacks: one adjoint launch over all nfields slices."""
    torch, sht, _lib, so = _gpu_env()
    lib = _lib.load()
    lmax, nlat, nlon, nf = 23, 24, 48, 4
    cfg = sht.create_gauss_config(lmax, nlat, nlon=nlon)
    oc = so.create_gauss_config(lmax, nlat, nlon=nlon)
    plan = cfg.plan(0)
    st = torch.cuda.current_stream(0).cuda_stream
    rng = np.random.default_rng(5)
    ybar = rng.standard_normal((nlat, nlon, nf))
    ws, n = _ws(torch, lib, plan, ANA, nf, F64, PREC_FP64)
    yd = sht.to_device(ybar, torch.float64, 0)
    abar = sht.julia_empty((lmax + 1, lmax + 1, nf), torch.complex128, "cuda:0")
    _lib.check(lib.shtb_synthesis_adjoint(plan.handle, yd.data_ptr(), abar.data_ptr(), nf, ws.data_ptr(), n, st),
               "adjoint")
    torch.cuda.synchronize()
    ref = np.stack([so.adjoint_synthesis(oc, ybar[:, :, k]) for k in range(nf)], axis=2)
    from _util import rel_l2, rand_alm
    assert rel_l2(sht.to_host(abar), ref) <= 1e-12

    A = rand_alm(lmax, lmax, nf, seed=21)
    ws, n = _ws(torch, lib, plan, SYN, nf, F64, PREC_FP64)
    Ad = sht.to_device(A, torch.complex128, 0)
    fbar = sht.julia_empty((nlat, nlon, nf), torch.float64, "cuda:0")
    _lib.check(lib.shtb_analysis_adjoint(plan.handle, Ad.data_ptr(), fbar.data_ptr(), nf, ws.data_ptr(), n, st),
               "adjoint")
    torch.cuda.synchronize()
    # the C entry returns the real projection of the analysis adjoint (the rrule's
    # ProjectTo onto the real field), ext/SHTnsKitAdvancedADExt.jl:95-112
    ref = np.stack([so.adjoint_analysis(oc, A[:, :, k]).real for k in range(nf)], axis=2)
    assert rel_l2(sht.to_host(fbar), ref) <= 1e-12
