"""
    SHTnsKitB200

GPU adapter for SHTnsKit.jl backed by `libshtb200.so` (B200, sm_100a). It registers
itself through SHTnsKit's vendor-neutral adapter protocol (src/device_utils.jl:8-99),
so `analysis(cfg, f::CuArray)`, `synthesis(cfg, alm::CuArray)` and the sphtor pair
route here. Load it *instead of* SHTnsKit's own CUDA extension: two adapters that both
recognise `CuArray` make SHTnsKit raise "multiple GPU adapters recognize ..."
(src/device_utils.jl:143-148); the reference extension is activated only when
KernelAbstractions is loaded as well, which this package does not need.

Every call goes through the library's C ABI (`include/shtb200.h`) with `ccall`;
there is no CPU fallback.
"""
module SHTnsKitB200

using CUDA
using SHTnsKit
import ChainRulesCore

const LIB = get(ENV, "SHTB200_LIB", joinpath(@__DIR__, "..", "..", "..", "shtb200", "libshtb200.so"))

const SHTB_F64 = Cint(0)
const SHTB_F32 = Cint(1)
const SHTB_PREC_FP64 = Cint(0)
const SHTB_PREC_MIXED = Cint(1)
const OP_SYN, OP_ANA, OP_SYN_V, OP_ANA_V = Cint(0), Cint(1), Cint(2), Cint(3)

struct B200Adapter end
const ADAPTER = B200Adapter()

function __init__()
    SHTnsKit._register_gpu_adapter!(:b200, ADAPTER)
    return nothing
end

# ---------------------------------------------------------------- adapter protocol
SHTnsKit._gpu_adapter_functional(::B200Adapter) = CUDA.functional() && isfile(LIB)
SHTnsKit._gpu_adapter_matches(::B200Adapter, ::CUDA.AnyCuArray) = true
SHTnsKit._gpu_adapter_matches(a::B200Adapter, x::AbstractArray) = (p = parent(x)) !== x && SHTnsKit._gpu_adapter_matches(a, p)
SHTnsKit._gpu_adapter_adapt(::B200Adapter, x) = CuArray(x)
SHTnsKit._gpu_adapter_dense(::B200Adapter, x::AbstractArray) = x isa CuArray ? x : (similar(x, eltype(x), size(x)) .= x)
SHTnsKit._allocation_device(a::CuArray) = CUDA.device(a)
SHTnsKit._on_allocation_device(f, d::CUDA.CuDevice) = d == CUDA.device() ? f() : CUDA.device!(f, d)
SHTnsKit.on_device(::CuArray) = SHTnsKit.GPU()

# ---------------------------------------------------------------- errors
function check(rc::Cint, op::Symbol)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:shtb_last_error, LIB), Cstring, ()))
    rc == -2 && throw(DimensionMismatch(msg))
    rc in (-1, -3, -8) && throw(ArgumentError(msg))
    throw(SHTnsKit.BackendUnavailableError(op, "$msg (status $rc)"))
end

# ---------------------------------------------------------------- plans (cached per cfg and device)
mutable struct Plan
    ptr::Ptr{Cvoid}
end
const PLANS = Dict{Tuple{UInt,Int,Float64},Plan}()
const PLANS_LOCK = ReentrantLock()

function plan(cfg::SHTnsKit.SHTConfig)
    key = (objectid(cfg), CUDA.deviceid(CUDA.device()), SHTnsKit.phi_inv_scale(cfg))
    lock(PLANS_LOCK) do
        get!(PLANS, key) do
            scale = SHTnsKit._uses_canonical_convention(cfg) ? C_NULL :
                    pointer(SHTnsKit._ensure_norm_scale_matrix!(cfg))
            out = Ref{Ptr{Cvoid}}(C_NULL)
            rc = ccall((:shtb_plan_create, LIB), Cint,
                       (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Cint, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                        Cdouble, Cdouble, Cint),
                       out, cfg.lmax, cfg.mmax, cfg.mres, cfg.nlat, cfg.nlon, cfg.x, cfg.w, scale,
                       SHTnsKit.phi_inv_scale(cfg), SHTnsKit._analysis_phi_scale(cfg), cfg.robert_form)
            check(rc, :plan_create)
            p = Plan(out[])
            finalizer(p) do q
                q.ptr == C_NULL || ccall((:shtb_plan_destroy, LIB), Cint, (Ptr{Cvoid},), q.ptr)
            end
            p
        end
    end
end

SHTnsKit._gpu_adapter_clear_cache!(::B200Adapter) = lock(() -> empty!(PLANS), PLANS_LOCK)

workspace(p::Plan, op, nf, dtype, prec) =
    CuArray{UInt8}(undef, max(256, ccall((:shtb_workspace_bytes, LIB), Csize_t,
                                         (Ptr{Cvoid}, Cint, Cint, Cint, Cint), p.ptr, op, nf, dtype, prec)))

stream() = CUDA.stream().handle
dtype_of(::Type{<:Union{Float64,ComplexF64}}) = SHTB_F64
dtype_of(::Type{<:Union{Float32,ComplexF32}}) = SHTB_F32
prec_of(T) = dtype_of(T) == SHTB_F64 ? SHTB_PREC_FP64 : SHTB_PREC_MIXED

# ---------------------------------------------------------------- transforms (3-D = batch)
function _synthesis(cfg, alm::CuArray{Complex{T}}; lcap::Int=cfg.lmax) where {T<:Union{Float32,Float64}}
    nf = size(alm, 3)
    f = CuArray{T}(undef, cfg.nlat, cfg.nlon, nf)
    p = plan(cfg)
    ws = workspace(p, OP_SYN, nf, dtype_of(T), prec_of(T))
    check(ccall((:shtb_synthesis, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, alm, f, nf, lcap, dtype_of(T), prec_of(T), ws, sizeof(ws), stream()), :synthesis)
    return f
end

function _analysis(cfg, f::CuArray{T}; lcap::Int=cfg.lmax) where {T<:Union{Float32,Float64}}
    nf = size(f, 3)
    alm = CuArray{Complex{T}}(undef, cfg.lmax + 1, cfg.mmax + 1, nf)
    p = plan(cfg)
    ws = workspace(p, OP_ANA, nf, dtype_of(T), prec_of(T))
    check(ccall((:shtb_analysis, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, f, alm, nf, lcap, dtype_of(T), prec_of(T), ws, sizeof(ws), stream()), :analysis)
    return alm
end

as3(x::CuArray) = ndims(x) == 3 ? x : reshape(x, size(x, 1), size(x, 2), 1)
drop3(x, like) = ndims(like) == 3 ? x : reshape(x, size(x, 1), size(x, 2))

function SHTnsKit._gpu_adapter_synthesis(::B200Adapter, cfg::SHTnsKit.SHTConfig, alm;
                                         real_output::Bool=true, use_rfft::Bool=false,
                                         fft_scratch=nothing, lcap::Int=cfg.lmax)
    fft_scratch === nothing || throw(ArgumentError("CUDA scalar transforms do not accept a host fft_scratch"))
    use_rfft && !real_output && throw(ArgumentError("use_rfft=true implies real_output"))
    real_output || throw(SHTnsKit.BackendUnavailableError(:synthesis, "real_output=false is not implemented by this backend"))
    size(alm, 1) == cfg.lmax + 1 && size(alm, 2) == cfg.mmax + 1 || throw(DimensionMismatch(
        "coefficients must have size ($(cfg.lmax + 1), $(cfg.mmax + 1)), got $(size(alm))"))
    a = alm isa CuArray{<:Complex} ? alm : CuArray{ComplexF64}(alm)
    return drop3(_synthesis(cfg, as3(a); lcap), alm)
end

function SHTnsKit._gpu_adapter_analysis(::B200Adapter, cfg::SHTnsKit.SHTConfig, f;
                                        use_rfft::Bool=false, fft_scratch=nothing, lcap::Int=cfg.lmax)
    fft_scratch === nothing || throw(ArgumentError("CUDA scalar transforms do not accept a host fft_scratch"))
    eltype(f) <: Real || throw(SHTnsKit.BackendUnavailableError(:analysis, "complex fields are not implemented by this backend"))
    size(f, 1) == cfg.nlat && size(f, 2) == cfg.nlon || throw(DimensionMismatch(
        "field must have size ($(cfg.nlat), $(cfg.nlon)), got $(size(f))"))
    return drop3(_analysis(cfg, as3(f); lcap), f)
end

function SHTnsKit._gpu_adapter_synthesis_sphtor(::B200Adapter, cfg::SHTnsKit.SHTConfig, S, T;
                                                real_output::Bool=true, use_rfft::Bool=false, lcap::Int=cfg.lmax)
    real_output || throw(SHTnsKit.BackendUnavailableError(:synthesis_sphtor, "real_output=false is not implemented"))
    S3, T3 = as3(CuArray{ComplexF64}(S)), as3(CuArray{ComplexF64}(T))
    nf = size(S3, 3)
    Vt = CuArray{Float64}(undef, cfg.nlat, cfg.nlon, nf); Vp = similar(Vt)
    p = plan(cfg)
    ws = workspace(p, OP_SYN_V, nf, SHTB_F64, SHTB_PREC_FP64)
    check(ccall((:shtb_synthesis_sphtor, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint,
                 CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, S3, T3, Vt, Vp, nf, lcap, SHTB_F64, SHTB_PREC_FP64, ws, sizeof(ws), stream()), :synthesis_sphtor)
    return drop3(Vt, S), drop3(Vp, S)
end

function SHTnsKit._gpu_adapter_analysis_sphtor(::B200Adapter, cfg::SHTnsKit.SHTConfig, Vt, Vp;
                                               use_rfft::Bool=false, lcap::Int=cfg.lmax)
    A, B = as3(CuArray{Float64}(Vt)), as3(CuArray{Float64}(Vp))
    nf = size(A, 3)
    S = CuArray{ComplexF64}(undef, cfg.lmax + 1, cfg.mmax + 1, nf); T = similar(S)
    p = plan(cfg)
    ws = workspace(p, OP_ANA_V, nf, SHTB_F64, SHTB_PREC_FP64)
    check(ccall((:shtb_analysis_sphtor, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint,
                 CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, A, B, S, T, nf, lcap, SHTB_F64, SHTB_PREC_FP64, ws, sizeof(ws), stream()), :analysis_sphtor)
    return drop3(S, Vt), drop3(T, Vt)
end

# batched entry points of the reference's CUDA extension (ext/SHTnsKitGPUExt.jl:1845-1975)
SHTnsKit.synthesis_batch(cfg::SHTnsKit.SHTConfig, alm::CuArray{<:Complex,3}; lcap::Int=cfg.lmax, kwargs...) =
    _synthesis(cfg, alm; lcap)
SHTnsKit.analysis_batch(cfg::SHTnsKit.SHTConfig, f::CuArray{<:Real,3}; lcap::Int=cfg.lmax, kwargs...) =
    _analysis(cfg, f; lcap)

# ---------------------------------------------------------------- packed LM layout (src/transforms.jl:125-227)
function _synthesis_packed(cfg, Q::CuVector{Complex{T}}, lcap::Int) where {T<:Union{Float32,Float64}}
    length(Q) == cfg.nlm || throw(DimensionMismatch("Qlm must have length $(cfg.nlm)"))
    f = CuArray{T}(undef, cfg.nlat, cfg.nlon)
    p = plan(cfg)
    ws = workspace(p, OP_SYN, 1, dtype_of(T), prec_of(T))
    check(ccall((:shtb_synthesis_packed, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, Q, f, 1, lcap, dtype_of(T), prec_of(T), ws, sizeof(ws), stream()), :synthesis_packed)
    return vec(f)
end

function _analysis_packed(cfg, Vr::CuVector{T}, lcap::Int) where {T<:Union{Float32,Float64}}
    length(Vr) == cfg.nlat * cfg.nlon || throw(DimensionMismatch("Vr must have length $(cfg.nlat * cfg.nlon)"))
    Q = CuArray{Complex{T}}(undef, cfg.nlm)
    p = plan(cfg)
    ws = workspace(p, OP_ANA, 1, dtype_of(T), prec_of(T))
    check(ccall((:shtb_analysis_packed, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, Vr, Q, 1, lcap, dtype_of(T), prec_of(T), ws, sizeof(ws), stream()), :analysis_packed)
    return Q
end

SHTnsKit.synthesis_packed(cfg::SHTnsKit.SHTConfig, Q::CuVector{<:Complex}) = _synthesis_packed(cfg, Q, cfg.lmax)
SHTnsKit.synthesis_packed_l(cfg::SHTnsKit.SHTConfig, Q::CuVector{<:Complex}, ltr::Integer) =
    _synthesis_packed(cfg, Q, Int(ltr))
SHTnsKit.analysis_packed(cfg::SHTnsKit.SHTConfig, Vr::CuVector{<:Real}) = _analysis_packed(cfg, Vr, cfg.lmax)
SHTnsKit.analysis_packed_l(cfg::SHTnsKit.SHTConfig, Vr::CuVector{<:Real}, ltr::Integer) =
    _analysis_packed(cfg, Vr, Int(ltr))

# ---------------------------------------------------------------- diagonal spectral operators
# (src/sphtor_transforms.jl:744-930, ext/GPUCommon.jl:1501-1512); `out` may be `in` itself
const SPEC_NEG_LL = Cint(0)
const SPEC_INV_NEG_LL = Cint(1)
function _spectral_op!(cfg, op::Cint, out::CuMatrix{Complex{T}}, in::CuMatrix{Complex{T}}) where {T<:Union{Float32,Float64}}
    expected = (cfg.lmax + 1, cfg.mmax + 1)
    size(in) == expected || throw(DimensionMismatch("spectral input dims"))
    size(out) == size(in) || throw(DimensionMismatch("spectral output dims"))
    check(ccall((:shtb_spectral_op, LIB), Cint,
                (Ptr{Cvoid}, Cint, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Ptr{Cvoid}),
                plan(cfg).ptr, op, in, out, 1, dtype_of(T), stream()), :spectral_op)
    return out
end
SHTnsKit.divergence_from_spheroidal!(cfg::SHTnsKit.SHTConfig, d::CuMatrix, S::CuMatrix) = _spectral_op!(cfg, SPEC_NEG_LL, d, S)
SHTnsKit.vorticity_from_toroidal!(cfg::SHTnsKit.SHTConfig, z::CuMatrix, T::CuMatrix) = _spectral_op!(cfg, SPEC_NEG_LL, z, T)
SHTnsKit.spheroidal_from_divergence!(cfg::SHTnsKit.SHTConfig, S::CuMatrix, d::CuMatrix) = _spectral_op!(cfg, SPEC_INV_NEG_LL, S, d)
SHTnsKit.toroidal_from_vorticity!(cfg::SHTnsKit.SHTConfig, T::CuMatrix, z::CuMatrix) = _spectral_op!(cfg, SPEC_INV_NEG_LL, T, z)
SHTnsKit.divergence_from_spheroidal(cfg::SHTnsKit.SHTConfig, S::CuMatrix) = _spectral_op!(cfg, SPEC_NEG_LL, similar(S), S)
SHTnsKit.vorticity_from_toroidal(cfg::SHTnsKit.SHTConfig, T::CuMatrix) = _spectral_op!(cfg, SPEC_NEG_LL, similar(T), T)
SHTnsKit.spheroidal_from_divergence(cfg::SHTnsKit.SHTConfig, d::CuMatrix) = _spectral_op!(cfg, SPEC_INV_NEG_LL, similar(d), d)
SHTnsKit.toroidal_from_vorticity(cfg::SHTnsKit.SHTConfig, z::CuMatrix) = _spectral_op!(cfg, SPEC_INV_NEG_LL, similar(z), z)
SHTnsKit.gpu_apply_laplacian!(cfg::SHTnsKit.SHTConfig, a::CuMatrix; device=SHTnsKit.GPU()) =
    _spectral_op!(cfg, SPEC_NEG_LL, a, a)

# ---------------------------------------------------------------- adjoint kernels behind the rrules
function _adjoint(sym::Symbol, op::Cint, cfg, ins::Tuple, outs::Tuple, nf)
    p = plan(cfg)
    ws = workspace(p, op, nf, SHTB_F64, SHTB_PREC_FP64)
    args = (p.ptr, ins..., outs..., Cint(nf), ws, Csize_t(sizeof(ws)), stream())
    rc = if length(ins) == 1
        ccall((sym, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}), args...)
    else
        ccall((sym, LIB), Cint, (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, CuPtr{Cvoid},
                                 Csize_t, Ptr{Cvoid}), args...)
    end
    check(rc, sym)
end

function ChainRulesCore.rrule(::typeof(SHTnsKit.synthesis), cfg::SHTnsKit.SHTConfig, alm::CuArray{ComplexF64,2};
                              real_output::Bool=true, kwargs...)
    f = SHTnsKit.synthesis(cfg, alm; real_output, kwargs...)
    function pullback(fbar)
        ybar = as3(CuArray{Float64}(ChainRulesCore.unthunk(fbar)))
        abar = CuArray{ComplexF64}(undef, cfg.lmax + 1, cfg.mmax + 1, 1)
        _adjoint(:shtb_synthesis_adjoint, OP_ANA, cfg, (ybar,), (abar,), 1)
        return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), reshape(abar, size(alm))
    end
    return f, pullback
end

function ChainRulesCore.rrule(::typeof(SHTnsKit.analysis), cfg::SHTnsKit.SHTConfig, f::CuArray{Float64,2}; kwargs...)
    alm = SHTnsKit.analysis(cfg, f; kwargs...)
    function pullback(abar)
        a = as3(CuArray{ComplexF64}(ChainRulesCore.unthunk(abar)))
        fbar = CuArray{Float64}(undef, cfg.nlat, cfg.nlon, 1)
        _adjoint(:shtb_analysis_adjoint, OP_SYN, cfg, (a,), (fbar,), 1)
        return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), reshape(fbar, size(f))
    end
    return alm, pullback
end

function ChainRulesCore.rrule(::typeof(SHTnsKit.synthesis_sphtor), cfg::SHTnsKit.SHTConfig,
                              S::CuArray{ComplexF64,2}, T::CuArray{ComplexF64,2}; kwargs...)
    V = SHTnsKit.synthesis_sphtor(cfg, S, T; kwargs...)
    function pullback(Vbar)
        z() = CUDA.zeros(Float64, cfg.nlat, cfg.nlon)
        vt = ChainRulesCore.unthunk(Vbar[1]); vp = ChainRulesCore.unthunk(Vbar[2])
        vt = vt isa ChainRulesCore.AbstractZero ? z() : CuArray{Float64}(vt)
        vp = vp isa ChainRulesCore.AbstractZero ? z() : CuArray{Float64}(vp)
        Sb = CuArray{ComplexF64}(undef, size(S)..., 1); Tb = similar(Sb)
        _adjoint(:shtb_synthesis_sphtor_adjoint, OP_ANA_V, cfg, (as3(vt), as3(vp)), (Sb, Tb), 1)
        return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), reshape(Sb, size(S)), reshape(Tb, size(T))
    end
    return V, pullback
end

function ChainRulesCore.rrule(::typeof(SHTnsKit.analysis_sphtor), cfg::SHTnsKit.SHTConfig,
                              Vt::CuArray{Float64,2}, Vp::CuArray{Float64,2}; kwargs...)
    ST = SHTnsKit.analysis_sphtor(cfg, Vt, Vp; kwargs...)
    function pullback(STbar)
        z() = CUDA.zeros(ComplexF64, cfg.lmax + 1, cfg.mmax + 1)
        sb = ChainRulesCore.unthunk(STbar[1]); tb = ChainRulesCore.unthunk(STbar[2])
        sb = sb isa ChainRulesCore.AbstractZero ? z() : CuArray{ComplexF64}(sb)
        tb = tb isa ChainRulesCore.AbstractZero ? z() : CuArray{ComplexF64}(tb)
        vt = CuArray{Float64}(undef, cfg.nlat, cfg.nlon, 1); vp = similar(vt)
        _adjoint(:shtb_analysis_sphtor_adjoint, OP_SYN_V, cfg, (as3(sb), as3(tb)), (vt, vp), 1)
        return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), reshape(vt, size(Vt)), reshape(vp, size(Vp))
    end
    return ST, pullback
end

end # module
