"""
    FFTAB200

GPU drop-in for FFTA.jl's complex and real transform path on one B200: the
plans, `mul!`, `*` and `size` of FFTA (src/plan.jl) on `CuArray`s, executed by
the C-ABI library `libfftab200.so` (sm_100a kernels; include/fftab200.h).

Element types are ComplexF32/ComplexF64 (and Float32/Float64 for the real
transforms); any other element type throws `ArgumentError` -- there is no CPU
fallback.  The argument checks and their messages are FFTA's own
(src/plan.jl:157-285), so code written against FFTA sees the same exceptions.
Host `Array`s go through [`plan_fft_host`](@ref) / [`plan_bfft_host`](@ref),
which stage the data through the library's pinned copy path.

The library is found at `ENV["FFTAB200_LIB"]`, else at
`ffta.jl_b200/libfftab200.so` of the repository this package lives in.
"""
module FFTAB200

using AbstractFFTs
using CUDA
using LinearAlgebra
import AbstractFFTs: plan_fft, plan_bfft, plan_rfft, plan_brfft, plan_inv

export plan_fft_host, plan_bfft_host, autotune!

const libfftab200 = get(ENV, "FFTAB200_LIB",
                        normpath(joinpath(@__DIR__, "..", "..", "..", "ffta.jl_b200",
                                          "libfftab200.so")))

# Status codes and constants of include/fftab200.h
const FB_OK, FB_ERR_DIMENSION_MISMATCH, FB_ERR_ARGUMENT, FB_ERR_DOMAIN = 0, 1, 2, 3
const FB_ERR_CUDA, FB_ERR_UNSUPPORTED, FB_ERR_OUT_OF_MEMORY = 4, 5, 6
const FB_C32, FB_C64 = Cint(0), Cint(1)
const FB_FORWARD, FB_BACKWARD = Cint(-1), Cint(1)
const DEFAULT_BLUESTEIN_CUTOFF = 73            # FFTA src/callgraph.jl:44

fbtype(::Type{ComplexF32}) = FB_C32
fbtype(::Type{ComplexF64}) = FB_C64
fbtype(::Type{Float32}) = FB_C32
fbtype(::Type{Float64}) = FB_C64
fbtype(::Type{T}) where {T} = throw(ArgumentError(
    "element type $T is not supported: only ComplexF32/ComplexF64 (and Float32/Float64) " *
    "run on the GPU, and there is no CPU fallback"))

last_error() = unsafe_string(ccall((:fb_last_error, libfftab200), Cstring, ()))

"Map a library status to the exception FFTA throws in the same situation."
function check(rc::Integer)
    rc == FB_OK && return nothing
    msg = last_error()
    rc == FB_ERR_DIMENSION_MISMATCH && throw(DimensionMismatch(msg))
    rc == FB_ERR_ARGUMENT && throw(ArgumentError(msg))
    rc == FB_ERR_DOMAIN && throw(DomainError(msg))
    rc == FB_ERR_OUT_OF_MEMORY && throw(OutOfMemoryError())
    rc == FB_ERR_UNSUPPORTED && throw(ArgumentError(msg))
    error("libfftab200: " * msg)
end

# ------------------------------------------------------------- complex plans
"""
A complex plan (FFTA's `FFTAPlan_cx`, src/plan.jl:9-20): the transform sizes,
the sorted region and the direction.  The device schedule is made once per
array layout (shape and strides of input and output) on first use.
"""
mutable struct GPUPlan_cx{T<:Complex,N,R} <: AbstractFFTs.Plan{T}
    sizes::NTuple{N,Int}
    region::R
    dir::Cint
    cutoff::Int
    flags::UInt32
    host::Bool                               # plans for host Arrays
    handles::Dict{Any,Ptr{Cvoid}}
    pinv::AbstractFFTs.Plan{T}
    function GPUPlan_cx{T,N,R}(sizes, region, dir, cutoff, flags, host) where {T,N,R}
        p = new{T,N,R}(sizes, region, dir, cutoff, flags, host, Dict{Any,Ptr{Cvoid}}())
        finalizer(p) do q
            for h in values(q.handles)
                ccall((:fb_plan_destroy, libfftab200), Cint, (Ptr{Cvoid},), h)
            end
            empty!(q.handles)
        end
        p
    end
end

# Base.size (src/plan.jl:36-47)
function Base.size(p::GPUPlan_cx{T,N}, i::Int) where {T,N}
    i < 1 && throw(DomainError(i, "No non-positive dimensions"))
    i > N ? 1 : p.sizes[i]
end
Base.size(p::GPUPlan_cx{T,N}) where {T,N} = ntuple(i -> size(p, i), Val(N))

_sortregion(r::Integer) = Int(r)
_sortregion(r::Tuple) = Tuple(sort!(collect(Int, r)))
_sortregion(r) = issorted(r) ? copy(r) : sort(r)
_regionlist(r) = r isa Integer ? [Int(r)] : collect(Int, r)

# _plan_fft (src/plan.jl:77-100)
function _plan(x::AbstractArray{T}, region, dir::Cint, host::Bool;
               BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, flags::Integer=0,
               _kwargs...) where {T}
    fbtype(T)
    T <: Complex || throw(ArgumentError("complex plans take complex arrays; use plan_rfft"))
    r = _sortregion(region)
    regs = _regionlist(r)
    all(d -> 1 <= d <= ndims(x), regs) ||
        throw(DimensionMismatch("Plan region is outside array dimensions."))
    sizes = Tuple(size(x, d) for d in regs)
    any(<=(0), sizes) && throw(DimensionMismatch("Array length must be strictly positive"))
    GPUPlan_cx{T,length(sizes),typeof(r)}(sizes, r, dir, BLUESTEIN_CUTOFF, UInt32(flags), host)
end

const CuComplex = Union{ComplexF32,ComplexF64}
plan_fft(x::CuArray{T}, region; kw...) where {T<:CuComplex} = _plan(x, region, FB_FORWARD, false; kw...)
plan_bfft(x::CuArray{T}, region; kw...) where {T<:CuComplex} = _plan(x, region, FB_BACKWARD, false; kw...)
# AbstractFFTs promotes real arrays to complex before planning; other element
# types are refused (no CPU fallback)
plan_fft(x::CuArray{T}, region; kw...) where {T} = (fbtype(T); throw(ArgumentError(
    "plan_fft takes ComplexF32/ComplexF64 arrays; convert real input with complex()")))
plan_bfft(x::CuArray{T}, region; kw...) where {T} = (fbtype(T); throw(ArgumentError(
    "plan_bfft takes ComplexF32/ComplexF64 arrays; convert real input with complex()")))

"Plans for host `Array`s: the library copies in, transforms and copies out."
plan_fft_host(x::Array{<:Complex}, region=1:ndims(x); kw...) = _plan(x, region, FB_FORWARD, true; kw...)
plan_bfft_host(x::Array{<:Complex}, region=1:ndims(x); kw...) = _plan(x, region, FB_BACKWARD, true; kw...)

# ifft = the backward plan scaled (AbstractFFTs' ScaledPlan)
function plan_inv(p::GPUPlan_cx{T,N,R}) where {T,N,R}
    q = GPUPlan_cx{T,N,R}(p.sizes, p.region, -p.dir, p.cutoff, p.flags, p.host)
    AbstractFFTs.ScaledPlan(q, AbstractFFTs.normalization(real(T), p.sizes, 1:N))
end

_strides(x) = Int64[strides(x)...]

function handle(p::GPUPlan_cx{T}, y::AbstractArray, x::AbstractArray) where {T}
    key = (size(x), strides(x), strides(y))
    get!(p.handles, key) do
        h = Ref{Ptr{Cvoid}}(C_NULL)
        dims = Int64[size(x)...]
        reg = Int32[_regionlist(p.region)...]
        check(ccall((:fb_plan_create_nd, libfftab200), Cint,
                    (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Cint,
                     Ptr{Int32}, Int64, UInt32),
                    h, fbtype(T), p.dir, ndims(x), dims, _strides(x), _strides(y), length(reg),
                    reg, p.cutoff, p.flags))
        h[]
    end
end

function _execute!(p::GPUPlan_cx, y::AbstractArray, x::AbstractArray)
    h = handle(p, y, x)
    if p.host
        GC.@preserve x y check(ccall((:fb_execute_host, libfftab200), Cint,
                                     (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                                     h, pointer(x), pointer(y), C_NULL))
    else
        stream = CUDA.stream().handle
        GC.@preserve x y check(ccall((:fb_execute, libfftab200), Cint,
                                     (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}),
                                     h, pointer(x), pointer(y), stream))
    end
    y
end

_region_isvalid_nd(r::Integer, N) = r == N == 1
_region_isvalid_nd(r, N) = length(r) == N && all(i -> r[i] == i, 1:N)
function _region_isvalid_md(r, M)
    length(r) == M || return false
    v = collect(r)
    all(i -> v[i] < v[i+1], 1:length(v)-1)
end

# mul! with FFTA's checks and messages
function LinearAlgebra.mul!(y::AbstractArray{T,N}, p::GPUPlan_cx{T,M}, x::AbstractArray{T,N}) where {T,N,M}
    Base.require_one_based_indexing(x, y)
    if M == 1
        # 1D plan on a vector (src/plan.jl:157-167) or an N-D array (:170-192)
        axes(x) == axes(y) || throw(DimensionMismatch(
            "input array has axes $(axes(x)), but output array has axes $(axes(y))"))
        if N == 1
            size(p) == size(x) || throw(DimensionMismatch(
                "plan has axes $(size(p)), but input array has axes $(size(x))"))
        else
            R1 = only(_regionlist(p.region))
            plen, xlen = size(p, 1), size(x, R1)
            plen == xlen || throw(DimensionMismatch(
                "plan has size $plen, but input array has size $xlen along region $R1"))
        end
    elseif M == N
        # ND plan, ND array (src/plan.jl:210-222)
        size(y) == size(x) || throw(DimensionMismatch(
            "input array has axes $(axes(x)), but output array has axes $(axes(y))"))
        size(p) == size(x) || throw(DimensionMismatch(
            "plan has size $(size(p)), but input array has size $(size(x))"))
        _region_isvalid_nd(p.region, N) ||
            throw(DimensionMismatch("Plan region is outside array dimensions."))
    else
        # M-dim plan on an N-dim array (src/plan.jl:260-272)
        size(y) == size(x) || throw(DimensionMismatch(
            "input array has axes $(axes(x)), but output array has axes $(axes(y))"))
        _region_isvalid_md(p.region, M) || throw(DimensionMismatch("Region is invalid."))
        r = _regionlist(p.region)
        (M > N || first(r) < 1 || last(r) > N) &&
            throw(DimensionMismatch("Plan region is outside array dimensions."))
        all(k -> size(p, k) == size(x, r[k]), 1:M) || throw(DimensionMismatch(
            "plan has size $(size(p)), but input array has size $(size(x))"))
    end
    isempty(x) && return y
    _execute!(p, y, x)
end

# Base.:* (src/plan.jl:374-384)
Base.:*(p::GPUPlan_cx{T}, x::AbstractArray{T}) where {T} = mul!(similar(x), p, x)

"""
    autotune!(p, x; iters=5)

Time the plan's candidate launch shapes on `x` (and a scratch output) and
keep the fastest for this layout (`fb_plan_autotune`); results do not change.
"""
function autotune!(p::GPUPlan_cx, x::AbstractArray; iters::Integer=5)
    y = similar(x)
    h = handle(p, y, x)
    stream = p.host ? C_NULL : CUDA.stream().handle
    GC.@preserve x y check(ccall((:fb_plan_autotune, libfftab200), Cint,
                                 (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint),
                                 h, pointer(x), pointer(y), stream, iters))
    p
end

# ---------------------------------------------------------------- real plans
"""
A real plan (FFTA's `FFTAPlan_re`, src/plan.jl:22-34): rfft (real input,
`flen ÷ 2 + 1` outputs along the first region dim) or brfft of length `flen`.
Only 1-D and 2-D regions, as in FFTA.
"""
mutable struct GPUPlan_re{T,N,R} <: AbstractFFTs.Plan{T}
    sizes::NTuple{N,Int}
    region::R
    dir::Cint
    flen::Int
    cutoff::Int
    handles::Dict{Any,Ptr{Cvoid}}
    pinv::AbstractFFTs.Plan{T}
    function GPUPlan_re{T,N,R}(sizes, region, dir, flen, cutoff) where {T,N,R}
        p = new{T,N,R}(sizes, region, dir, flen, cutoff, Dict{Any,Ptr{Cvoid}}())
        finalizer(p) do q
            for h in values(q.handles)
                ccall((:fb_plan_destroy, libfftab200), Cint, (Ptr{Cvoid},), h)
            end
            empty!(q.handles)
        end
        p
    end
end

function Base.size(p::GPUPlan_re{T,N}, i::Int) where {T,N}
    i < 1 && throw(DomainError(i, "No non-positive dimensions"))
    i > N ? 1 : (i == 1 ? p.flen : p.sizes[i])
end
Base.size(p::GPUPlan_re{T,N}) where {T,N} = ntuple(i -> size(p, i), Val(N))

function plan_rfft(x::CuArray{T}, region; BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF,
                   _kw...) where {T<:Union{Float32,Float64}}
    r = _sortregion(region)
    length(_regionlist(r)) > 2 && throw(ArgumentError("only supports 1D and 2D FFTs"))
    sizes = Tuple(size(x, d) for d in _regionlist(r))
    GPUPlan_re{Complex{T},length(sizes),typeof(r)}(sizes, r, FB_FORWARD, sizes[1],
                                                   BLUESTEIN_CUTOFF)
end

function plan_brfft(x::CuArray{T}, len::Integer, region;
                    BLUESTEIN_CUTOFF=DEFAULT_BLUESTEIN_CUTOFF, _kw...) where {T<:CuComplex}
    r = _sortregion(region)
    length(_regionlist(r)) > 2 && throw(ArgumentError("only supports 1D and 2D FFTs"))
    sizes = Tuple(d == first(_regionlist(r)) ? Int(len) : size(x, d) for d in _regionlist(r))
    GPUPlan_re{T,length(sizes),typeof(r)}(sizes, r, FB_BACKWARD, Int(len), BLUESTEIN_CUTOFF)
end

function real_handle(p::GPUPlan_re, realdims::Dims, precision::Type)
    get!(p.handles, realdims) do
        h = Ref{Ptr{Cvoid}}(C_NULL)
        dims = Int64[realdims...]
        reg = Int32[_regionlist(p.region)...]
        check(ccall((:fb_plan_create_real, libfftab200), Cint,
                    (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Ptr{Int64}, Cint, Ptr{Int32}, Int64,
                     UInt32),
                    h, fbtype(precision), p.dir, length(dims), dims, length(reg), reg,
                    p.cutoff, 0))
        h[]
    end
end

# rfft (src/plan.jl:390-454 vector, :506-513 1-D plan on arrays, :532-542 2-D)
function Base.:*(p::GPUPlan_re{Complex{T}}, x::CuArray{T}) where {T<:Union{Float32,Float64}}
    p.dir == FB_FORWARD || throw(ArgumentError(
        "only FFT_FORWARD supported for real $(ndims(x) == 1 ? "vectors" : "arrays")"))
    r = _regionlist(p.region)
    (first(r) < 1 || last(r) > ndims(x)) &&
        throw(DimensionMismatch("Plan region is outside array dimensions."))
    got = Tuple(size(x, d) for d in r)
    got == size(p) || throw(DimensionMismatch(
        "plan has size $(size(p)), but input array has size $got"))
    ydims = ntuple(d -> d == first(r) ? size(x, d) ÷ 2 + 1 : size(x, d), ndims(x))
    y = CuArray{Complex{T}}(undef, ydims)
    isempty(x) && throw(DimensionMismatch("Array length must be strictly positive"))
    h = real_handle(p, size(x), T)
    GC.@preserve x y check(ccall((:fb_execute, libfftab200), Cint,
                                 (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}),
                                 h, pointer(x), pointer(y), CUDA.stream().handle))
    y
end

# brfft (src/plan.jl:456-504, :515-527, :544-583)
function Base.:*(p::GPUPlan_re{T}, x::CuArray{T}) where {T<:CuComplex}
    p.dir == FB_BACKWARD || throw(ArgumentError(
        "only FFT_BACKWARD supported for complex $(ndims(x) == 1 ? "vectors" : "arrays")"))
    r = _regionlist(p.region)
    (first(r) < 1 || last(r) > ndims(x)) &&
        throw(DimensionMismatch("Plan region is outside array dimensions."))
    rlen = p.flen ÷ 2 + 1
    size(x, first(r)) == rlen || throw(DimensionMismatch(
        "real $(length(r))D plan has size $(p.flen). Dimension of input array along region " *
        "$(first(r)) should have size $rlen, but has size $(size(x, first(r)))"))
    ydims = ntuple(d -> d == first(r) ? p.flen : size(x, d), ndims(x))
    y = CuArray{real(T)}(undef, ydims)
    h = real_handle(p, ydims, real(T))
    GC.@preserve x y check(ccall((:fb_execute, libfftab200), Cint,
                                 (Ptr{Cvoid}, CuPtr{Cvoid}, CuPtr{Cvoid}, Ptr{Cvoid}),
                                 h, pointer(x), pointer(y), CUDA.stream().handle))
    y
end

version() = unsafe_string(ccall((:fb_version, libfftab200), Cstring, ()))

end # module
