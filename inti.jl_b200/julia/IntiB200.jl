"""
    IntiB200

Julia side of libinti_b200.so: B200 (sm_100a) application of Inti.jl's
integral operators through `ccall`.  It plugs into Inti the way the FMM
extension does (ext/IntiFMM3DExt.jl:12-33): node arrays are repacked as
`Matrix{Float64}(dim, n)`, and the operator comes back as a
`LinearMaps.LinearMap` whose `mul!` calls the library.

    using Inti, IntiB200
    S, D = IntiB200.single_double_layer(; op, target = Q, source = Q,
                                         compression = (method = :b200, precision = :fp64),
                                         correction = (method = :dim,))
    σ, stats = IntiB200.gmres(I / 2 + D + S, rhs; rtol = 1e-10, mode = :mixed)
    # or, from an existing Inti operator: IntiB200.assemble_b200(iop; correction = δD)

The C ABI is declared in include/inti_b200.h.  Julia was not available where
this package was developed; the entry points it calls are exercised from
Python (ctypes) by the repository's tests.  Package dependencies: Inti,
LinearMaps and ChainRulesCore (the reverse rule of `A * σ`).
"""
module IntiB200

using LinearAlgebra
using SparseArrays
using LinearMaps
using ChainRulesCore
import Inti

const LIB = get(ENV, "INTI_B200_LIB", joinpath(@__DIR__, "..", "_build", "libinti_b200.so"))

const LAPLACE, HELMHOLTZ = Cint(0), Cint(1)
const SL, DL, ADL, HS = Cint(0), Cint(1), Cint(2), Cint(3)
const FP64, FP32C = Cint(0), Cint(1)
const F64, C128 = Cint(0), Cint(1)

struct B200Error <: Exception
    code::Int
    msg::String
end
Base.showerror(io::IO, e::B200Error) = print(io, "libinti_b200 error ", e.code, ": ", e.msg)

function check(status, ctx_ptr = C_NULL)
    status == 0 && return nothing
    msg = unsafe_string(ccall((:inti_last_error, LIB), Cstring, (Ptr{Cvoid},), ctx_ptr))
    # the same split as the reference's error types
    status == 1 && throw(ArgumentError(msg))
    status == 2 && throw(DimensionMismatch(msg))
    throw(B200Error(status, msg))
end

# ----------------------------------------------------------------------------
# handles
# ----------------------------------------------------------------------------
mutable struct Context
    ptr::Ptr{Cvoid}
    function Context(device::Integer = 0)
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:inti_ctx_create, LIB), Cint, (Cint, Ptr{Cvoid}, Ref{Ptr{Cvoid}}), device, C_NULL, out))
        c = new(out[])
        finalizer(c -> ccall((:inti_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), c.ptr), c)
        return c
    end
end

const DEFAULT = Ref{Union{Nothing,Context}}(nothing)
default_context() = something(DEFAULT[], (DEFAULT[] = Context(0)))

mutable struct QuadHandle
    ptr::Ptr{Cvoid}
    ctx::Context
    n::Int
    dim::Int
end

"""
    upload(Q; ctx) -> QuadHandle

Copy a quadrature's nodes, normals and weights (src/quadrature.jl:7-11) to
the device.  Elements are the columns of `etype2qtags` (contiguous blocks).
"""
function upload(Q::Inti.Quadrature{N}; ctx = default_context()) where {N}
    n = length(Q)
    X = Matrix{Float64}(undef, N, n)
    Nrm = Matrix{Float64}(undef, N, n)
    W = Vector{Float64}(undef, n)
    has_normals = true
    for (j, q) in enumerate(Q.qnodes)
        X[:, j] = q.coords
        W[j] = q.weight
        if q.normal === nothing
            has_normals = false
        else
            Nrm[:, j] = q.normal
        end
    end
    nq = length(Q.etype2qtags) == 1 ? size(first(values(Q.etype2qtags)), 1) : 0
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve X Nrm W begin
        check(ccall((:inti_quad_create, LIB), Cint,
                    (Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Ref{Ptr{Cvoid}}),
                    ctx.ptr, N, n, X, has_normals ? Nrm : C_NULL, W, nq, out), ctx.ptr)
    end
    h = QuadHandle(out[], ctx, n, N)
    finalizer(h -> ccall((:inti_quad_destroy, LIB), Cint, (Ptr{Cvoid},), h.ptr), h)
    return h
end

"""Plain target points (`Vector{SVector}`), as `coords(::SVector)` allows
(src/quadrature.jl:50)."""
function upload(pts::AbstractVector{<:AbstractVector}; ctx = default_context())
    N = length(first(pts))
    X = reduce(hcat, pts)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve X check(ccall((:inti_quad_create, LIB), Cint,
        (Ptr{Cvoid}, Cint, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Ref{Ptr{Cvoid}}),
        ctx.ptr, N, length(pts), X, C_NULL, C_NULL, 0, out), ctx.ptr)
    h = QuadHandle(out[], ctx, length(pts), N)
    finalizer(h -> ccall((:inti_quad_destroy, LIB), Cint, (Ptr{Cvoid},), h.ptr), h)
    return h
end

mutable struct CsrHandle
    ptr::Ptr{Cvoid}
    ctx::Context
end

"""A `SparseMatrixCSC` correction (src/bdim.jl:193-194) on the device; the
1-based CSC arrays are transposed to CSR by the library, pattern intact."""
function upload(A::SparseMatrixCSC{T}; ctx = default_context()) where {T<:Union{Float64,ComplexF64}}
    m, n = size(A)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    colptr = Vector{Int64}(A.colptr)
    rowval = Vector{Int64}(A.rowval)
    nz = A.nzval
    GC.@preserve colptr rowval nz check(ccall((:inti_csr_create_from_csc, LIB), Cint,
        (Ptr{Cvoid}, Int64, Int64, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Cvoid}, Cint, Ref{Ptr{Cvoid}}),
        ctx.ptr, m, n, length(nz), colptr, rowval, nz, T <: Complex ? C128 : F64, out), ctx.ptr)
    h = CsrHandle(out[], ctx)
    finalizer(h -> ccall((:inti_csr_destroy, LIB), Cint, (Ptr{Cvoid},), h.ptr), h)
    return h
end

# ----------------------------------------------------------------------------
# operators
# ----------------------------------------------------------------------------
pde_code(::Inti.Laplace) = LAPLACE
pde_code(::Inti.Helmholtz) = HELMHOLTZ
wavenumber(op::Inti.Helmholtz) = complex(op.k)
wavenumber(::Inti.Laplace) = 0.0im
kernel_code(::Inti.SingleLayerKernel) = SL
kernel_code(::Inti.DoubleLayerKernel) = DL
kernel_code(::Inti.AdjointDoubleLayerKernel) = ADL
kernel_code(::Inti.HyperSingularKernel) = HS

mutable struct OpHandle
    ptr::Ptr{Cvoid}
    keep::Tuple  # quadratures and correction outlive the operator
end

function op_handle(K, tgt::QuadHandle, src::QuadHandle, corr, precision::Symbol)
    op = Inti.operator(K)
    k = wavenumber(op)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:inti_op_create, LIB), Cint,
                (Ptr{Cvoid}, Cint, Cint, Float64, Float64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ref{Ptr{Cvoid}}),
                src.ctx.ptr, pde_code(op), kernel_code(K), real(k), imag(k), tgt.ptr, src.ptr,
                corr === nothing ? C_NULL : corr.ptr, precision == :fp32c ? FP32C : FP64, out), src.ctx.ptr)
    h = OpHandle(out[], (tgt, src, corr))
    finalizer(h -> ccall((:inti_op_destroy, LIB), Cint, (Ptr{Cvoid},), h.ptr), h)
    return h
end

"""
    B200Map{T} <: LinearMap{T}

A device operator as a `LinearMap`: `mul!(y, A, x, α, β)` is one
`inti_op_apply` (the role of the FunctionMap closure in
ext/IntiFMM3DExt.jl:28-33), so the reference's lazy sums
(`I/2 + D - im*k*S`, src/api.jl:179-184) compose with it unchanged.
"""
struct B200Map{T} <: LinearMaps.LinearMap{T}
    h::OpHandle
    m::Int
    n::Int
    ctx::Context
end
Base.size(A::B200Map) = (A.m, A.n)

function apply!(y::AbstractVector, A::B200Map{T}, x::AbstractVector, α = true, β = false) where {T}
    xx = Vector{T}(x)
    yy = y isa Vector{T} ? y : Vector{T}(y)
    a = Float64[real(α), imag(complex(α))]
    b = Float64[real(β), imag(complex(β))]
    GC.@preserve xx yy a b check(ccall((:inti_op_apply, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Cvoid}, Int64, Int32, Ptr{Float64}, Ptr{Float64}, Cint),
        A.h.ptr, xx, A.n, yy, A.m, 1, a, b, 0), A.ctx.ptr)
    yy === y || copyto!(y, yy)
    return y
end
LinearMaps._unsafe_mul!(y::AbstractVector, A::B200Map, x::AbstractVector) = apply!(y, A, x)
LinearMaps._unsafe_mul!(y::AbstractVector, A::B200Map, x::AbstractVector, α::Number, β::Number) =
    apply!(y, A, x, α, β)

# Many columns in one call: from 8 columns on, FP64 3D operators (every
# kernel) evaluate each kernel value once for up to 64 columns.
function apply!(Y::AbstractMatrix, A::B200Map{T}, X::AbstractMatrix, α = true, β = false) where {T}
    XX = Matrix{T}(X)
    YY = Y isa Matrix{T} ? Y : Matrix{T}(Y)
    a = Float64[real(α), imag(complex(α))]
    b = Float64[real(β), imag(complex(β))]
    GC.@preserve XX YY a b check(ccall((:inti_op_apply, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Cvoid}, Int64, Int32, Ptr{Float64}, Ptr{Float64}, Cint),
        A.h.ptr, XX, size(XX, 1), YY, size(YY, 1), size(XX, 2), a, b, 0), A.ctx.ptr)
    YY === Y || copyto!(Y, YY)
    return Y
end
LinearMaps._unsafe_mul!(Y::AbstractMatrix, A::B200Map, X::AbstractMatrix) = apply!(Y, A, X)
LinearMaps._unsafe_mul!(Y::AbstractMatrix, A::B200Map, X::AbstractMatrix, α::Number, β::Number) =
    apply!(Y, A, X, α, β)

"""
    transpose_apply(A::B200Map, x) -> transpose(A) * x

`inti_op_apply_transpose`: the product with the (unconjugated) transpose,
correction rows included.
"""
function transpose_apply(A::B200Map{T}, x::AbstractVector) where {T}
    xx = Vector{T}(x)
    yy = zeros(T, A.n)
    a, b = Float64[1, 0], Float64[0, 0]
    GC.@preserve xx yy a b check(ccall((:inti_op_apply_transpose, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Cvoid}, Int64, Int32, Ptr{Float64}, Ptr{Float64}, Cint),
        A.h.ptr, xx, A.m, yy, A.n, 1, a, b, 0), A.ctx.ptr)
    return yy
end

"""
    grad_sources(A::B200Map{Float64}, ū, σ)

Cotangents of `σ` and of the source quadrature (coordinates `dim × n`,
normals `dim × n`, weights `n`) for `u = A σ` with `∂J/∂u = ū`, from the
hand-written adjoint kernel (`inti_op_grad_sources`, Laplace single and
double layer, FP64): kernel tiles are recomputed, nothing `m × n` is stored.
The pair terms only; a correction is not part of it.
"""
function grad_sources(A::B200Map{Float64}, ubar::AbstractVector, σ::AbstractVector)
    src = A.h.keep[2]::QuadHandle
    g, s = Vector{Float64}(ubar), Vector{Float64}(σ)
    dσ, dw = zeros(A.n), zeros(A.n)
    dx, dn = zeros(src.dim, A.n), zeros(src.dim, A.n)
    GC.@preserve g s dσ dx dn dw check(ccall((:inti_op_grad_sources, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Cint),
        A.h.ptr, g, s, dσ, dx, dn, dw, 0), A.ctx.ptr)
    return (σ = dσ, coords = dx, normals = dn, weights = dw)
end

"""
    ChainRulesCore.rrule(::typeof(*), A::B200Map, σ)

Reverse rule of the device product `u = A * σ` (Inti.jl itself only
differentiates forward, through ForwardDiff: src/reference_interpolation.jl:
36-39).  The pullback maps `ū` to `Aᴴ ū` for `σ` (the transpose apply,
conjugated for complex operators, correction rows included) and, for real
Laplace single and double layers, to a `Tangent` of the operator holding the
source-geometry cotangents `coords`, `normals`, `weights` from the adjoint
kernel.  A DIM correction is held constant: its dependence on the geometry
is not differentiated.
"""
function ChainRulesCore.rrule(::typeof(*), A::B200Map{T}, σ::AbstractVector) where {T}
    u = A * σ
    function b200_pullback(ū)
        ubar = unthunk(ū)
        if T <: Complex
            return NoTangent(), NoTangent(), conj.(transpose_apply(A, conj.(ubar)))
        end
        dσ = transpose_apply(A, ubar)
        g = try
            grad_sources(A, ubar, σ)
        catch err
            err isa B200Error || rethrow()
            nothing  # kernels without source gradients (ADL, HS, FP32C)
        end
        g === nothing && return NoTangent(), NoTangent(), dσ
        Ā = Tangent{typeof(A)}(; coords = g.coords, normals = g.normals, weights = g.weights)
        return NoTangent(), Ā, dσ
    end
    return u, b200_pullback
end

"""
    set_symmetric!(ctx, flag)

Square operators created afterwards use (`true`, the default) or skip the
symmetric pair kernel, which evaluates each unordered node pair once for both
products.
"""
set_symmetric!(ctx::Context, flag::Bool) =
    check(ccall((:inti_ctx_set_symmetric, LIB), Cint, (Ptr{Cvoid}, Cint), ctx.ptr, flag), ctx.ptr)

"""
    set_partial_budget!(ctx, bytes)

Bytes of partial sums a symmetric operator created afterwards may hold
(default 2e9; `0` restores it).  Larger operators run their work in panels,
so their memory stays O(N) plus the budget; `panels(A)` reports the count.
"""
set_partial_budget!(ctx::Context, bytes::Real) =
    check(ccall((:inti_ctx_set_partial_budget, LIB), Cint, (Ptr{Cvoid}, Float64), ctx.ptr, bytes), ctx.ptr)
panels(A::B200Map) = Int(ccall((:inti_op_panels, LIB), Cint, (Ptr{Cvoid},), A.h.ptr))

"""
    set_single_launch!(ctx, flag)

Small FP64 operators (at most 2^20 pairs, 65,536 sources) created afterwards apply with one
kernel launch per product (`true`, the default) or with the tiled kernels;
`single_launch(A)` reports the form of an operator.
"""
set_single_launch!(ctx::Context, flag::Bool) =
    check(ccall((:inti_ctx_set_single_launch, LIB), Cint, (Ptr{Cvoid}, Cint), ctx.ptr, flag), ctx.ptr)
single_launch(A::B200Map) = ccall((:inti_op_single_launch, LIB), Cint, (Ptr{Cvoid},), A.h.ptr) == 1

"""
    set_gmres_small!(ctx, max_unknowns)

GMRES on systems of at most `max_unknowns` unknowns (default 8192) runs each
Arnoldi step in one single-CTA kernel and checks the residual every four
steps; `0` turns that form off.
"""
set_gmres_small!(ctx::Context, max_unknowns::Integer) =
    check(ccall((:inti_ctx_set_gmres_small, LIB), Cint, (Ptr{Cvoid}, Int64), ctx.ptr, max_unknowns), ctx.ptr)

"""
    set_shard!(A::B200Map, rank, nranks)

One process per GPU: `A` computes only rank `rank`'s share of the node pairs
(a symmetric operator), so `mul!` returns a partial product and the sum over
the ranks (one `MPI.Allreduce!`) is the whole; rank 0 carries the correction
and `β*y`. `nranks = 1` restores the whole operator.
"""
set_shard!(A::B200Map, rank::Integer, nranks::Integer) =
    check(ccall((:inti_op_set_shard, LIB), Cint, (Ptr{Cvoid}, Cint, Cint), A.h.ptr, rank, nranks), A.ctx.ptr)

as_linearmap(h::OpHandle, ::Type{T}, m, n, ctx) where {T} = B200Map{T}(h, m, n, ctx)

"""
    assemble_b200(iop::Inti.IntegralOperator; precision = :fp64, correction = nothing)

The GPU counterpart of `assemble_matrix`/`assemble_fmm` (src/nystrom.jl:
103-169): a matrix-free `LinearMap` evaluated on the fly.
"""
function assemble_b200(iop::Inti.IntegralOperator; precision = :fp64, correction = nothing,
                       ctx = default_context())
    tgt = upload(Inti.target(iop); ctx)
    # one handle for target === source: the library then uses its symmetric pair kernel
    src = Inti.source(iop) === Inti.target(iop) ? tgt : upload(Inti.source(iop); ctx)
    corr = correction === nothing ? nothing : upload(correction; ctx)
    h = op_handle(Inti.kernel(iop), tgt, src, corr, precision)
    return as_linearmap(h, eltype(iop), size(iop)..., ctx)
end

"""
    bdim_correction_b200(op, Q; green_multiplier = -0.5, derivative = false)

`(δS, δD)` of src/bdim.jl:50-196 for `target === source`, built on the GPU
and returned as device handles.
"""
function bdim_correction_b200(op, Q::QuadHandle; green_multiplier = nothing, derivative = false)
    k = wavenumber(op)
    dS = Ref{Ptr{Cvoid}}(C_NULL)
    dD = Ref{Ptr{Cvoid}}(C_NULL)
    gm = green_multiplier === nothing ? C_NULL : Vector{Float64}(green_multiplier)
    GC.@preserve gm check(ccall((:inti_dim_correction, LIB), Cint,
        (Ptr{Cvoid}, Cint, Float64, Float64, Ptr{Cvoid}, Cint, Ptr{Cvoid}, Ref{Ptr{Cvoid}}, Ref{Ptr{Cvoid}}),
        Q.ctx.ptr, pde_code(op), real(k), imag(k), Q.ptr, derivative, gm, dS, dD), Q.ctx.ptr)
    hS, hD = CsrHandle(dS[], Q.ctx), CsrHandle(dD[], Q.ctx)
    for h in (hS, hD)
        finalizer(h -> ccall((:inti_csr_destroy, LIB), Cint, (Ptr{Cvoid},), h.ptr), h)
    end
    return hS, hD
end

"""
    bdim_correction_b200(op, target::QuadHandle, Q::QuadHandle; green_multiplier, maxdist = Inf,
                         derivative = false)

The same for targets other than the source nodes (src/api.jl:105-148): every
target within `maxdist` of its nearest source node is corrected through that
node's element (src/quadrature.jl:264-286).  `green_multiplier` holds one
value per target (`_green_multiplier` of src/nystrom.jl:196-207).
"""
function bdim_correction_b200(op, target::QuadHandle, Q::QuadHandle; green_multiplier, maxdist = Inf,
                              derivative = false)
    k = wavenumber(op)
    dS = Ref{Ptr{Cvoid}}(C_NULL)
    dD = Ref{Ptr{Cvoid}}(C_NULL)
    gm = Vector{Float64}(green_multiplier)
    GC.@preserve gm check(ccall((:inti_dim_correction_targets, LIB), Cint,
        (Ptr{Cvoid}, Cint, Float64, Float64, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}, Float64,
         Ref{Ptr{Cvoid}}, Ref{Ptr{Cvoid}}),
        Q.ctx.ptr, pde_code(op), real(k), imag(k), target.ptr, Q.ptr, derivative, gm, Float64(maxdist), dS, dD),
        Q.ctx.ptr)
    hS, hD = CsrHandle(dS[], Q.ctx), CsrHandle(dD[], Q.ctx)
    for h in (hS, hD)
        finalizer(h -> ccall((:inti_csr_destroy, LIB), Cint, (Ptr{Cvoid},), h.ptr), h)
    end
    return hS, hD
end

"""
    single_double_layer(; op, target, source, compression, correction, derivative = false)

Mirror of `Inti.single_double_layer` (src/api.jl:65-187) for
`compression = (method = :b200, precision = :fp64 | :fp32c)` and
`correction = (method = :dim, [target_location | green_multiplier], [maxdist])`
or `(method = :none,)`.  Returns
`S = A_S + δS`, `D = A_D + δD` as LinearMaps (the correction applied in the
same device pass).
"""
function single_double_layer(; op, target, source, compression = (method = :b200,),
                             correction = (method = :dim,), derivative = false, ctx = default_context())
    compression.method == :b200 ||
        throw(ArgumentError("Unknown compression.method $(compression.method). Available options: (:b200,)"))
    precision = get(compression, :precision, :fp64)
    G = derivative ? Inti.AdjointDoubleLayerKernel(op) : Inti.SingleLayerKernel(op)
    dG = derivative ? Inti.HyperSingularKernel(op) : Inti.DoubleLayerKernel(op)
    tgt = upload(target; ctx)
    src = target === source ? tgt : upload(source; ctx)
    cS = cD = nothing
    if correction.method == :dim && target === source
        μ = haskey(correction, :green_multiplier) ? correction.green_multiplier : nothing
        cS, cD = bdim_correction_b200(op, src; green_multiplier = μ, derivative)
    elseif correction.method == :dim
        # src/utils.jl:200-228: target_location or green_multiplier, not both
        haskey(correction, :target_location) || haskey(correction, :green_multiplier) ||
            throw(ArgumentError("missing target_location field in correction"))
        (haskey(correction, :target_location) && haskey(correction, :green_multiplier)) &&
            throw(ArgumentError("conflicting target_location and green_multiplier fields in correction"))
        haskey(correction, :maxdist) || @warn("missing maxdist field in correction: setting to Inf")
        μ = haskey(correction, :green_multiplier) ? correction.green_multiplier :
            fill(Inti._green_multiplier(correction.target_location), length(target))
        cS, cD = bdim_correction_b200(op, tgt, src; green_multiplier = μ,
                                      maxdist = get(correction, :maxdist, Inf), derivative)
    elseif correction.method != :none
        throw(ArgumentError("Unknown correction.method $(correction.method). Available options: (:dim, :none)"))
    end
    T = Inti.default_kernel_eltype(op)
    m, n = length(target), length(source)
    S = as_linearmap(op_handle(G, tgt, src, cS, precision), T, m, n, ctx)
    D = as_linearmap(op_handle(dG, tgt, src, cD, precision), T, m, n, ctx)
    return S, D
end

"""
    gmres(L, b; rtol = 1e-10, restart = 100, maxiter = 1000, mode = :fp64)

GMRES on the device for `L = λI + Σ cₜ Aₜ` built from `B200Map`s with
LinearMaps' `+`, scalar `*` and `I` (the operators of
docs/src/examples/poisson.jl:160-168 and helmholtz_scattering.jl:485-495).
`mode = :mixed` runs FP32 inner solves refined against FP64 residuals.
Returns `(x, stats::NamedTuple)`.
"""
function gmres(L::LinearMaps.LinearMap, b::AbstractVector; rtol = 1e-10, restart = 100, maxiter = 1000,
               mode = :fp64)
    shift = Ref(0.0im)
    terms = Tuple{ComplexF64,B200Map}[]
    collect_terms!(L, 1.0 + 0im, shift, terms)
    isempty(terms) && throw(ArgumentError("L has no device operator"))
    ctx = terms[1][2].ctx
    T = eltype(L)
    bb = Vector{T}(b)
    x = zeros(T, length(bb))
    ops = Ptr{Cvoid}[t[2].h.ptr for t in terms]
    coefs = reduce(vcat, [Float64[real(c), imag(c)] for (c, _) in terms])
    sh = Float64[real(shift[]), imag(shift[])]
    stats = zeros(UInt8, 48)  # inti_gmres_stats: 6 Int32 + 3 Float64
    GC.@preserve ops coefs sh bb x stats check(ccall((:inti_gmres, LIB), Cint,
        (Ptr{Cvoid}, Int32, Ptr{Ptr{Cvoid}}, Ptr{Float64}, Ptr{Float64}, Ptr{Cvoid}, Ptr{Cvoid}, Float64,
         Int32, Int32, Int32, Cint, Ptr{Float64}, Ptr{UInt8}),
        ctx.ptr, length(ops), ops, coefs, sh, bb, x, rtol, restart, maxiter, mode == :mixed ? 1 : 0, 0,
        C_NULL, stats), ctx.ptr)
    ints = reinterpret(Int32, stats[1:24])
    flts = reinterpret(Float64, stats[25:48])
    return x, (iterations = ints[1], outer = ints[2], fp64_applies = ints[3], fp32_applies = ints[4],
               converged = ints[5] == 1, relres = flts[1], seconds = flts[2], setup_seconds = flts[3])
end

collect_terms!(A::B200Map, c, shift, terms) = push!(terms, (ComplexF64(c), A))
collect_terms!(A::LinearMaps.UniformScalingMap, c, shift, terms) = (shift[] += c * A.λ; terms)
collect_terms!(A::LinearMaps.ScaledMap, c, shift, terms) = collect_terms!(A.lmap, c * A.λ, shift, terms)
function collect_terms!(A::LinearMaps.LinearCombination, c, shift, terms)
    foreach(M -> collect_terms!(M, c, shift, terms), A.maps)
    return terms
end
collect_terms!(A, c, shift, terms) = throw(ArgumentError("unsupported term $(typeof(A)) in a device GMRES"))

end # module
