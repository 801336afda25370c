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

# Arithmetic path of a call. The rule is explicit: Float64/ComplexF64 arrays run the plain
# FP64 path (relative L2 <= 1e-12 against the reference CPU result); Float32/ComplexF32
# arrays run the mixed path (`precision = :mixed`: Legendre contraction as fp16x3 tensor-core
# products with FP32 accumulation, relative L2 <= 1e-6, measured 2e-7..4e-7 at lmax 1023),
# which is at least as accurate as a plain Float32 recurrence. `precision = :fp64` on Float32
# arrays promotes them to Float64 for the call and rounds the result back.
function precision_of(::Type{T}, precision::Symbol) where {T}
    precision === :auto && return dtype_of(T) == SHTB_F64 ? SHTB_PREC_FP64 : SHTB_PREC_MIXED
    precision === :fp64 && return SHTB_PREC_FP64
    precision === :mixed && return SHTB_PREC_MIXED
    throw(ArgumentError("precision must be :auto, :fp64 or :mixed, got :$precision"))
end

# ---------------------------------------------------------------- transforms (3-D = batch)
# Writes into `f` (nlat, nlon, nf), real of the precision's element type.
function _synthesis!(f::CuArray{T,3}, cfg, alm::CuArray{Complex{T},3}, lcap::Int, prec::Cint) where {T}
    nf = size(alm, 3)
    p = plan(cfg)
    ws = workspace(p, OP_SYN, nf, dtype_of(T), prec)
    check(ccall((:shtb_synthesis, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, alm, f, nf, lcap, dtype_of(T), prec, ws, sizeof(ws), stream()), :synthesis)
    return f
end

function _analysis!(alm::CuArray{Complex{T},3}, cfg, f::CuArray{T,3}, lcap::Int, prec::Cint) where {T}
    nf = size(f, 3)
    p = plan(cfg)
    ws = workspace(p, OP_ANA, nf, dtype_of(T), prec)
    check(ccall((:shtb_analysis, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, f, alm, nf, lcap, dtype_of(T), prec, ws, sizeof(ws), stream()), :analysis)
    return alm
end

# complex grids (FP64): synthesis with real_output = false, analysis of complex fields
function _synthesis_cplx!(g::CuArray{ComplexF64,3}, cfg, alm::CuArray{ComplexF64,3}, lcap::Int)
    nf = size(alm, 3)
    p = plan(cfg)
    ws = workspace(p, OP_SYN, nf, SHTB_F64, SHTB_PREC_FP64)
    check(ccall((:shtb_synthesis_cplx, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, alm, g, nf, lcap, ws, sizeof(ws), stream()), :synthesis)
    return g
end

function _analysis_cplx!(alm::CuArray{ComplexF64,3}, cfg, g::CuArray{ComplexF64,3}, lcap::Int)
    nf = size(g, 3)
    p = plan(cfg)
    ws = workspace(p, OP_ANA, nf, SHTB_F64, SHTB_PREC_FP64)
    check(ccall((:shtb_analysis_cplx, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, g, alm, nf, lcap, ws, sizeof(ws), stream()), :analysis)
    return alm
end

as3(x::CuArray) = ndims(x) == 3 ? x : reshape(x, size(x, 1), size(x, 2), 1)
drop3(x, like) = ndims(like) == 3 ? x : reshape(x, size(x, 1), size(x, 2))
dense3(x, ::Type{T}) where {T} = as3(x isa CuArray{T} ? x : CuArray{T}(x))

check_spectral(cfg, alm) = size(alm, 1) == cfg.lmax + 1 && size(alm, 2) == cfg.mmax + 1 || throw(DimensionMismatch(
    "coefficients must have size ($(cfg.lmax + 1), $(cfg.mmax + 1)), got $(size(alm))"))
check_grid(cfg, f) = size(f, 1) == cfg.nlat && size(f, 2) == cfg.nlon || throw(DimensionMismatch(
    "field must have size ($(cfg.nlat), $(cfg.nlon)), got $(size(f))"))
check_lcap(cfg, lcap) = 0 <= lcap <= cfg.lmax || throw(ArgumentError("lcap must satisfy 0 ≤ lcap ≤ lmax=$(cfg.lmax)"))

# synthesis of any 2-D/3-D coefficient array: real grid of the precision's type, or a
# complex grid (real_output = false, FP64)
function synthesis_any(cfg, alm; real_output::Bool=true, use_rfft::Bool=false, lcap::Int=cfg.lmax,
                       precision::Symbol=:auto)
    use_rfft && !real_output && throw(ArgumentError("use_rfft=true implies real_output"))
    check_spectral(cfg, alm)
    check_lcap(cfg, lcap)
    if !real_output
        a = dense3(alm, ComplexF64)
        return drop3(_synthesis_cplx!(CuArray{ComplexF64}(undef, cfg.nlat, cfg.nlon, size(a, 3)), cfg, a, lcap), alm)
    end
    Tin = real(eltype(alm)) <: Float32 ? Float32 : Float64
    prec = precision_of(Tin, precision)
    T = prec == SHTB_PREC_FP64 ? Float64 : Float32
    a = dense3(alm, Complex{T})
    f = _synthesis!(CuArray{T}(undef, cfg.nlat, cfg.nlon, size(a, 3)), cfg, a, lcap, prec)
    return drop3(T === Tin ? f : CuArray{Tin}(f), alm)
end

# analysis of any 2-D/3-D grid: real fields on the precision's path, complex fields on FP64
function analysis_any(cfg, f; use_rfft::Bool=false, lcap::Int=cfg.lmax, precision::Symbol=:auto)
    check_grid(cfg, f)
    check_lcap(cfg, lcap)
    if eltype(f) <: Complex
        use_rfft && throw(ArgumentError("use_rfft=true requires a real-valued input"))
        g = dense3(f, ComplexF64)
        return drop3(_analysis_cplx!(CuArray{ComplexF64}(undef, cfg.lmax + 1, cfg.mmax + 1, size(g, 3)), cfg, g, lcap), f)
    end
    Tin = eltype(f) <: Float32 ? Float32 : Float64
    prec = precision_of(Tin, precision)
    T = prec == SHTB_PREC_FP64 ? Float64 : Float32
    x = dense3(f, T)
    alm = _analysis!(CuArray{Complex{T}}(undef, cfg.lmax + 1, cfg.mmax + 1, size(x, 3)), cfg, x, lcap, prec)
    return drop3(T === Tin ? alm : CuArray{Complex{Tin}}(alm), f)
end

function SHTnsKit._gpu_adapter_synthesis(::B200Adapter, cfg::SHTnsKit.SHTConfig, alm;
                                         real_output::Bool=true, use_rfft::Bool=false,
                                         fft_scratch=nothing, lcap::Int=cfg.lmax, precision::Symbol=:auto)
    fft_scratch === nothing || throw(ArgumentError("CUDA scalar transforms do not accept a host fft_scratch"))
    return synthesis_any(cfg, alm; real_output, use_rfft, lcap, precision)
end

function SHTnsKit._gpu_adapter_analysis(::B200Adapter, cfg::SHTnsKit.SHTConfig, f;
                                        use_rfft::Bool=false, fft_scratch=nothing, lcap::Int=cfg.lmax,
                                        precision::Symbol=:auto)
    fft_scratch === nothing || throw(ArgumentError("CUDA scalar transforms do not accept a host fft_scratch"))
    return analysis_any(cfg, f; use_rfft, lcap, precision)
end

function _synthesis_sphtor(cfg, S, T; real_output::Bool=true, lcap::Int=cfg.lmax)
    real_output || throw(SHTnsKit.BackendUnavailableError(:synthesis_sphtor, "real_output=false is not implemented"))
    check_spectral(cfg, S); check_spectral(cfg, T); check_lcap(cfg, lcap)
    S3, T3 = dense3(S, ComplexF64), dense3(T, ComplexF64)
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

function _analysis_sphtor(cfg, Vt, Vp; lcap::Int=cfg.lmax)
    check_grid(cfg, Vt); check_grid(cfg, Vp); check_lcap(cfg, lcap)
    A, B = dense3(Vt, Float64), dense3(Vp, Float64)
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

SHTnsKit._gpu_adapter_synthesis_sphtor(::B200Adapter, cfg::SHTnsKit.SHTConfig, S, T;
                                       real_output::Bool=true, use_rfft::Bool=false, lcap::Int=cfg.lmax) =
    _synthesis_sphtor(cfg, S, T; real_output, lcap)
SHTnsKit._gpu_adapter_analysis_sphtor(::B200Adapter, cfg::SHTnsKit.SHTConfig, Vt, Vp;
                                      use_rfft::Bool=false, lcap::Int=cfg.lmax) =
    _analysis_sphtor(cfg, Vt, Vp; lcap)

# ---------------------------------------------------------------- direct methods of the reference's CUDA extension
# batched scalar transforms (ext/SHTnsKitGPUExt.jl:1845-1975)
SHTnsKit.synthesis_batch(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, alm::CuArray{<:Complex,3};
                         real_output::Bool=true, use_rfft::Bool=false, lcap::Int=cfg.lmax, precision::Symbol=:auto) =
    synthesis_any(cfg, alm; real_output, use_rfft, lcap, precision)
SHTnsKit.synthesis_batch(cfg::SHTnsKit.SHTConfig, alm::CuArray{<:Complex,3}; kwargs...) =
    SHTnsKit.synthesis_batch(SHTnsKit.GPU(), cfg, alm; kwargs...)
SHTnsKit.synthesis_batch_cplx(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, alm::CuArray{<:Complex,3}) =
    synthesis_any(cfg, alm; real_output=false)
SHTnsKit.synthesis_batch_cplx(cfg::SHTnsKit.SHTConfig, alm::CuArray{<:Complex,3}) =
    synthesis_any(cfg, alm; real_output=false)
SHTnsKit.analysis_batch(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, f::CuArray{<:Real,3};
                        use_rfft::Bool=false, lcap::Int=cfg.lmax, precision::Symbol=:auto) =
    analysis_any(cfg, f; use_rfft, lcap, precision)
SHTnsKit.analysis_batch(cfg::SHTnsKit.SHTConfig, f::CuArray{<:Real,3}; kwargs...) =
    SHTnsKit.analysis_batch(SHTnsKit.GPU(), cfg, f; kwargs...)

# into caller-owned device outputs: the library writes `output` directly when it is a dense
# CuArray of the path's element type, else through a temporary
function _into!(output, result)
    result === output || copyto!(output, result)
    return output
end
function SHTnsKit.synthesis_batch!(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, output::CuArray{T,3},
                                   alm::CuArray{<:Complex,3}; real_output::Bool=true, use_rfft::Bool=false,
                                   lcap::Int=cfg.lmax, precision::Symbol=:auto) where {T}
    check_grid(cfg, output); check_spectral(cfg, alm); check_lcap(cfg, lcap)
    size(output, 3) == size(alm, 3) || throw(DimensionMismatch("output and coefficient batches differ"))
    if real_output && T <: Real
        prec = precision_of(T, precision)
        if (prec == SHTB_PREC_FP64 && T === Float64) || (prec == SHTB_PREC_MIXED && T === Float32)
            return _synthesis!(output, cfg, dense3(alm, Complex{T}), lcap, prec)
        end
    elseif !real_output && T === ComplexF64
        return _synthesis_cplx!(output, cfg, dense3(alm, ComplexF64), lcap)
    end
    !real_output && T <: Real && throw(ArgumentError("real plan output storage requires real_output=true"))
    return _into!(output, synthesis_any(cfg, alm; real_output, use_rfft, lcap, precision))
end
SHTnsKit.synthesis_batch!(cfg::SHTnsKit.SHTConfig, output::CuArray{<:Number,3}, alm::CuArray{<:Complex,3};
                          kwargs...) = SHTnsKit.synthesis_batch!(SHTnsKit.GPU(), cfg, output, alm; kwargs...)
function SHTnsKit.analysis_batch!(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, output::CuArray{Complex{T},3},
                                  f::CuArray{<:Number,3}; use_rfft::Bool=false, lcap::Int=cfg.lmax,
                                  precision::Symbol=:auto) where {T}
    check_grid(cfg, f); check_spectral(cfg, output); check_lcap(cfg, lcap)
    size(output, 3) == size(f, 3) || throw(DimensionMismatch("output and field batches differ"))
    if eltype(f) === T
        prec = precision_of(T, precision)
        if (prec == SHTB_PREC_FP64 && T === Float64) || (prec == SHTB_PREC_MIXED && T === Float32)
            return _analysis!(output, cfg, f, lcap, prec)
        end
    elseif eltype(f) === ComplexF64 && T === Float64
        return _analysis_cplx!(output, cfg, f, lcap)
    end
    return _into!(output, analysis_any(cfg, f; use_rfft, lcap, precision))
end
SHTnsKit.analysis_batch!(cfg::SHTnsKit.SHTConfig, output::CuArray{<:Complex,3}, f::CuArray{<:Number,3};
                         kwargs...) = SHTnsKit.analysis_batch!(SHTnsKit.GPU(), cfg, output, f; kwargs...)

# in-place single-field transforms, with a plan or a configuration (ext/SHTnsKitGPUExt.jl:1978-2020)
SHTnsKit.synthesis!(::SHTnsKit.GPU, plan::SHTnsKit.SHTPlan, output::CuArray{<:Number,2}, alm::CuArray{<:Complex,2};
                    real_output::Bool=true) =
    (SHTnsKit.synthesis_batch!(SHTnsKit.GPU(), plan.cfg, as3(output), as3(alm); real_output); output)
SHTnsKit.synthesis!(plan::SHTnsKit.SHTPlan, output::CuArray{<:Number,2}, alm::CuArray{<:Complex,2};
                    real_output::Bool=true) = SHTnsKit.synthesis!(SHTnsKit.GPU(), plan, output, alm; real_output)
SHTnsKit.analysis!(::SHTnsKit.GPU, plan::SHTnsKit.SHTPlan, output::CuArray{<:Complex,2}, f::CuArray{<:Number,2}) =
    (SHTnsKit.analysis_batch!(SHTnsKit.GPU(), plan.cfg, as3(output), as3(f)); output)
SHTnsKit.analysis!(plan::SHTnsKit.SHTPlan, output::CuArray{<:Complex,2}, f::CuArray{<:Number,2}) =
    SHTnsKit.analysis!(SHTnsKit.GPU(), plan, output, f)
function SHTnsKit.synthesis!(cfg::SHTnsKit.SHTConfig, output::CuArray{<:Number,2}, alm::CuArray{<:Complex,2};
                             real_output::Bool=true, fft_scratch=nothing, use_rfft::Bool=false)
    fft_scratch === nothing || throw(ArgumentError("CUDA scalar transforms do not accept fft_scratch"))
    SHTnsKit.synthesis_batch!(SHTnsKit.GPU(), cfg, as3(output), as3(alm); real_output, use_rfft)
    return output
end
function SHTnsKit.analysis!(cfg::SHTnsKit.SHTConfig, output::CuArray{<:Complex,2}, f::CuArray{<:Number,2};
                            fft_scratch=nothing, use_rfft::Bool=false)
    fft_scratch === nothing || throw(ArgumentError("CUDA scalar transforms do not accept fft_scratch"))
    SHTnsKit.analysis_batch!(SHTnsKit.GPU(), cfg, as3(output), as3(f); use_rfft)
    return output
end

# batched vector transforms (ext/SHTnsKitGPUExt.jl:1294-1315)
SHTnsKit.synthesis_sphtor_batch(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, S::CuArray{<:Complex,3},
                                T::CuArray{<:Complex,3}; real_output::Bool=true) =
    _synthesis_sphtor(cfg, S, T; real_output)
SHTnsKit.synthesis_sphtor_batch(cfg::SHTnsKit.SHTConfig, S::CuArray{<:Complex,3}, T::CuArray{<:Complex,3}; kwargs...) =
    SHTnsKit.synthesis_sphtor_batch(SHTnsKit.GPU(), cfg, S, T; kwargs...)
SHTnsKit.analysis_sphtor_batch(::SHTnsKit.GPU, cfg::SHTnsKit.SHTConfig, Vt::CuArray{<:Real,3}, Vp::CuArray{<:Real,3}) =
    _analysis_sphtor(cfg, Vt, Vp)
SHTnsKit.analysis_sphtor_batch(cfg::SHTnsKit.SHTConfig, Vt::CuArray{<:Real,3}, Vp::CuArray{<:Real,3}) =
    SHTnsKit.analysis_sphtor_batch(SHTnsKit.GPU(), cfg, Vt, Vp)

# in-place vector transforms with a plan (ext/SHTnsKitGPUExt.jl:1349-1364)
function SHTnsKit.analysis_sphtor!(plan::SHTnsKit.SHTPlan, Sout::CuArray, Tout::CuArray, Vt::CuArray, Vp::CuArray)
    S, T = _analysis_sphtor(plan.cfg, Vt, Vp)
    copyto!(Sout, S); copyto!(Tout, T)
    return Sout, Tout
end
function SHTnsKit.synthesis_sphtor!(plan::SHTnsKit.SHTPlan, Vt::CuArray, Vp::CuArray, S::CuArray, T::CuArray;
                                    real_output::Bool=true)
    A, B = _synthesis_sphtor(plan.cfg, S, T; real_output)
    copyto!(Vt, A); copyto!(Vp, B)
    return Vt, Vp
end

# ---------------------------------------------------------------- packed LM layout (src/transforms.jl:125-227)
function _synthesis_packed(cfg, Q::CuVector{Complex{T}}, lcap::Int) where {T<:Union{Float32,Float64}}
    length(Q) == cfg.nlm || throw(DimensionMismatch("Qlm must have length $(cfg.nlm)"))
    f = CuArray{T}(undef, cfg.nlat, cfg.nlon)
    p = plan(cfg)
    ws = workspace(p, OP_SYN, 1, dtype_of(T), precision_of(T, :auto))
    check(ccall((:shtb_synthesis_packed, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, Q, f, 1, lcap, dtype_of(T), precision_of(T, :auto), ws, sizeof(ws), stream()), :synthesis_packed)
    return vec(f)
end

function _analysis_packed(cfg, Vr::CuVector{T}, lcap::Int) where {T<:Union{Float32,Float64}}
    length(Vr) == cfg.nlat * cfg.nlon || throw(DimensionMismatch("Vr must have length $(cfg.nlat * cfg.nlon)"))
    Q = CuArray{Complex{T}}(undef, cfg.nlm)
    p = plan(cfg)
    ws = workspace(p, OP_ANA, 1, dtype_of(T), precision_of(T, :auto))
    check(ccall((:shtb_analysis_packed, LIB), Cint,
                (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Cint, Cint, Cint, Cint, CuPtr{Cvoid}, Csize_t, Ptr{Cvoid}),
                p.ptr, Vr, Q, 1, lcap, dtype_of(T), precision_of(T, :auto), ws, sizeof(ws), stream()), :analysis_packed)
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

# batch rrules (ext/SHTnsKitAdvancedADExt.jl:95-135): one adjoint launch over all nfields
# slices instead of a loop of per-slice adjoints
function ChainRulesCore.rrule(::typeof(SHTnsKit.synthesis_batch), cfg::SHTnsKit.SHTConfig,
                              alm::CuArray{ComplexF64,3}; real_output::Bool=true, use_rfft::Bool=false)
    real_output || throw(SHTnsKit.BackendUnavailableError(:synthesis_batch, "adjoint of real_output=false is not implemented"))
    f = SHTnsKit.synthesis_batch(cfg, alm; real_output, use_rfft)
    function pullback(fbar)
        fb = ChainRulesCore.unthunk(fbar)
        fb isa ChainRulesCore.AbstractZero && return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), ChainRulesCore.ZeroTangent()
        ybar = CuArray{Float64}(fb)
        nf = size(ybar, 3)
        abar = CuArray{ComplexF64}(undef, cfg.lmax + 1, cfg.mmax + 1, nf)
        _adjoint(:shtb_synthesis_adjoint, OP_ANA, cfg, (ybar,), (abar,), nf)
        return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), abar
    end
    return f, pullback
end

function ChainRulesCore.rrule(::typeof(SHTnsKit.analysis_batch), cfg::SHTnsKit.SHTConfig,
                              f::CuArray{Float64,3}; use_rfft::Bool=false)
    alm = SHTnsKit.analysis_batch(cfg, f; use_rfft)
    function pullback(abar)
        ab = ChainRulesCore.unthunk(abar)
        ab isa ChainRulesCore.AbstractZero && return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), ChainRulesCore.ZeroTangent()
        a = CuArray{ComplexF64}(ab)
        nf = size(a, 3)
        fbar = CuArray{Float64}(undef, cfg.nlat, cfg.nlon, nf)
        _adjoint(:shtb_analysis_adjoint, OP_SYN, cfg, (a,), (fbar,), nf)
        return ChainRulesCore.NoTangent(), ChainRulesCore.NoTangent(), fbar
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
