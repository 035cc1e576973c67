# CuLAMPB200.jl -- Julia ccall layer over libculamp_b200 (include/culamp.h).
#
# Drop-in for the kernelized path of CuLAMP.jl: the functions below keep the
# reference's names and signatures (src/solvers/SinkhornKernel.jl:477-489,
# src/solvers/MirrorProxKernel.jl:1019, src/solvers/AnnealedSinkhorn.jl:65-76)
# and forward device pointers of CuArray{Float64} to the C ABI. A 3 x N
# column-major CuArray has the point-major layout the library expects.
#
# Julia is not installed in the environment this library was built in, so this
# file has not been executed; it is the binding a maintainer adds next to
# CuLAMP.jl, whose run_dot / run_ctransfer call sites then dispatch here.
module CuLAMPB200

using CUDA
using ChainRulesCore
using LinearAlgebra: dot

const libculamp = joinpath(@__DIR__, "..", "libculamp_b200.so")

const CULAMP_FLAG_TRUE_PINF = UInt32(1)
const CULAMP_FLAG_CHECK_ALWAYS = UInt32(2)
const CULAMP_FLAG_MARGINAL_ONLY = UInt32(4)
const CULAMP_FLAG_FORM_PLAIN = UInt32(8)
const CULAMP_FLAG_NO_GRAPH = UInt32(16)
const CULAMP_FLAG_FEAT_X6 = UInt32(32)
const CULAMP_FLAG_FEAT_FP64 = UInt32(64)
const CULAMP_FLAG_FORM_FP32 = UInt32(128)
const CULAMP_FLAG_LADDER = UInt32(256)
const CULAMP_FLAG_FORM_FP64 = UInt32(512)
const CULAMP_FLAG_NO_PERSIST = UInt32(1024)

# struct culamp_args (EOTArgs, src/Utilities.jl:18-31)
struct CArgs
    eta_p::Float64; eta_mu::Float64; tau_p::Float64; tau_mu::Float64
    alpha::Float64; B::Float64; epsilon::Float64; anneal_mult::Float64
    itermax::Int64; inner_iter::Int64; tmax::Float64; verbose::Int32; pad::Int32
end
CArgs(a) = CArgs(a.eta_p, a.eta_mu, a.tau_p, a.tau_mu, a.alpha, a.B, Float64(a.epsilon),
                 a.anneal_mult, a.itermax, a.inner_iter, a.tmax, Int32(a.verbose), Int32(0))

struct CLogRow
    time_s::Float64; iter::Float64; infeas::Float64; ot_objective::Float64; primal::Float64; dual::Float64
end

mutable struct CStats
    iterations::Int64; num_iter::Int64; residual::Float64; objective::Float64; winf::Float64
    eta_t::Float64; s_t::Float64; elapsed_ms::Float64; log_rows::Int64; stopped::Int32; status::Int32
    CStats() = new(0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0, 0)
end

const _handle = Ref{Ptr{Cvoid}}(C_NULL)

function handle()
    if _handle[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:culamp_create, libculamp), Cint, (Ptr{Ptr{Cvoid}}, Cint), h, CUDA.device().handle)
        st == 0 || error("culamp_create failed with status $st")
        _handle[] = h[]
    end
    return _handle[]
end

function check(st)
    if st != 0
        msg = unsafe_string(ccall((:culamp_last_error, libculamp), Cstring, (Ptr{Cvoid},), handle()))
        error("culamp status $st: $msg")
    end
end

stream_ptr() = reinterpret(Ptr{Cvoid}, CUDA.stream().handle)

"""
    sinkhorn_color_transfer(img1, img2, marginal1, marginal2, args, frequency=100, p=2;
                            return_cuda=false, return_assignments=true, φ0=nothing, ψ0=nothing)

SinkhornKernel.jl:477-559 on libculamp_b200.
"""
function sinkhorn_color_transfer(img1::CuArray{Float64}, img2::CuArray{Float64},
                                 marginal1::CuArray{Float64}, marginal2::CuArray{Float64},
                                 args, frequency::Int=100, p::Union{Int,Float64}=2;
                                 return_cuda::Bool=false, return_assignments::Bool=true,
                                 φ0=nothing, ψ0=nothing, flags::UInt32=UInt32(0))
    d, N = size(img1)
    M = size(img2, 2)
    φ = CUDA.zeros(Float64, N)
    ψ = CUDA.zeros(Float64, M)
    stats = CStats()
    cargs = Ref(CArgs(args))
    logbuf = Vector{CLogRow}(undef, 100_000)
    st = ccall((:culamp_sinkhorn, libculamp), Cint,
               (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32, CuPtr{Float64},
                CuPtr{Float64}, Ptr{CArgs}, Int64, Float64, CuPtr{Float64}, CuPtr{Float64}, UInt32,
                CuPtr{Float64}, CuPtr{Float64}, Ref{CStats}, Ptr{CLogRow}, Int64, Ptr{Cvoid}),
               handle(), img1, img2, N, M, d, marginal1, marginal2, cargs, frequency, Float64(p),
               isnothing(φ0) ? CU_NULL : pointer(φ0), isnothing(ψ0) ? CU_NULL : pointer(ψ0), flags,
               φ, ψ, stats, logbuf, length(logbuf), stream_ptr())
    check(st)
    if args.verbose
        println("time(s),iter,infeas,ot_objective,dual")
        for r in logbuf[1:stats.log_rows]
            @printf "%.6e,%d,%.14e,%.14e,%.14e,sinkhorn_kernel\n" r.time_s Int(r.iter) r.infeas r.ot_objective r.dual
        end
    end
    if !return_assignments
        return_cuda && return φ, ψ, stats.objective, stats.residual, stats.num_iter
        return Array(φ), Array(ψ), stats.objective, stats.residual
    end
    out1 = similar(img1); out2 = similar(img2)
    cp = p == 1 ? 1.0 : 2.0   # the reference's barycentric map cost (SinkhornKernel.jl:146-150)
    check(ccall((:culamp_barycentric_sk, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32,
                 CuPtr{Float64}, CuPtr{Float64}, Float64, Float64, Float64, Ptr{Cvoid}),
                handle(), out1, img1, img2, N, M, d, φ, ψ, args.eta_p, stats.winf, cp, stream_ptr()))
    check(ccall((:culamp_barycentric_sk, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32,
                 CuPtr{Float64}, CuPtr{Float64}, Float64, Float64, Float64, Ptr{Cvoid}),
                handle(), out2, img2, img1, M, N, d, ψ, φ, args.eta_p, stats.winf, cp, stream_ptr()))
    return Array(φ), Array(ψ), Array(out1), Array(out2)
end

"""
    extragradient_color_transfer(img1, img2, marginal1, marginal2, args, frequency=100, p=2.0)

MirrorProxKernel.jl:1019-1132 (LAMP) on libculamp_b200; returns (ν, φ, ψ).
"""
function extragradient_color_transfer(img1::CuArray{Float64}, img2::CuArray{Float64},
                                      marginal1::CuArray{Float64}, marginal2::CuArray{Float64},
                                      args, frequency::Int=100, p::Float64=2.0; flags::UInt32=UInt32(0))
    d, N = size(img1)
    M = size(img2, 2)
    ν = CUDA.zeros(Float64, M); φ = CUDA.zeros(Float64, N)
    ψ = CUDA.zeros(Float64, M); θ = CUDA.zeros(Float64, M)
    stats = CStats()
    cargs = Ref(CArgs(args))
    logbuf = Vector{CLogRow}(undef, 100_000)
    check(ccall((:culamp_lamp, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32, CuPtr{Float64},
                 CuPtr{Float64}, Ptr{CArgs}, Int64, Float64, UInt32, CuPtr{Float64}, CuPtr{Float64},
                 CuPtr{Float64}, CuPtr{Float64}, Ref{CStats}, Ptr{CLogRow}, Int64, Ptr{Cvoid}),
                handle(), img1, img2, N, M, d, marginal1, marginal2, cargs, frequency, p, flags,
                ν, φ, ψ, θ, stats, logbuf, length(logbuf), stream_ptr()))
    return Array(ν), Array(φ), Array(ψ)
end

"""
    annealed_sinkhorn_euclidean(marginal1, marginal2, location1, location2, out1, out2,
                                potentials, args, frequency, p)

AnnealedSinkhorn.jl:65-177 on libculamp_b200 (potentials file output kept).
"""
function annealed_sinkhorn_euclidean(marginal1::CuArray{Float64}, marginal2::CuArray{Float64},
                                     location1::CuArray{Float64}, location2::CuArray{Float64},
                                     out1::String, out2::String, potentials::String, args,
                                     frequency::Int, p)
    d, N = size(location1)
    M = size(location2, 2)
    φ = CUDA.zeros(Float64, N); ψ = CUDA.zeros(Float64, M)
    stats = CStats()
    cargs = Ref(CArgs(args))
    check(ccall((:culamp_annealed_sinkhorn, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32, CuPtr{Float64},
                 CuPtr{Float64}, Ptr{CArgs}, Int64, Float64, UInt32, CuPtr{Float64}, CuPtr{Float64},
                 Ref{CStats}, Ptr{CLogRow}, Int64, Ptr{Cvoid}),
                handle(), location1, location2, N, M, d, marginal1, marginal2, cargs, frequency,
                Float64(p), UInt32(0), φ, ψ, stats, C_NULL, 0, stream_ptr()))
    φ_out, ψ_out = Array(φ), Array(ψ)
    if potentials != ""
        open(potentials * ".row", "w") do f; foreach(v -> println(f, v), φ_out); end
        open(potentials * ".col", "w") do f; foreach(v -> println(f, v), ψ_out); end
    end
    return φ_out, ψ_out, stats.objective
end

# ---------------------------------------------------------------- batched solves

struct CInstance
    x::CuPtr{Float64}; y::CuPtr{Float64}; r::CuPtr{Float64}; c::CuPtr{Float64}
    phi::CuPtr{Float64}; psi::CuPtr{Float64}; n::Int64; m::Int64; d::Int32; reserved::Int32
end

struct CBatchStats
    iterations::Int64; num_iter::Int64; residual::Float64; objective::Float64; winf::Float64
    stopped::Int32; status::Int32
end

mutable struct CBatchInfo
    elapsed_ms::Float64; tune_ms::Float64; target_ctas_per_sm::Int32; feat_tiles_per_unit::Int32
    unroll::Int32; launches_per_iteration::Int32; phases::Int32; reserved::Int32
    CBatchInfo() = new(0.0, 0.0, 0, 0, 0, 0, 0, 0)
end

"""
    batched_sinkhorn(xs, ys, rs, cs, args, frequency=100, p=2; flags=0)

Many independent kernel Sinkhorn problems (each as in sinkhorn_color_transfer,
SinkhornKernel.jl:477-559) of uneven sizes in one culamp_batched_sinkhorn call.
xs[k] is d x N_k, ys[k] d x M_k (CuArray{Float64}); returns (φs, ψs, stats).
"""
function batched_sinkhorn(xs, ys, rs, cs, args, frequency::Int=100, p=2; flags::UInt32=UInt32(0))
    K = length(xs)
    φs = [CUDA.zeros(Float64, size(xs[k], 2)) for k in 1:K]
    ψs = [CUDA.zeros(Float64, size(ys[k], 2)) for k in 1:K]
    insts = [CInstance(pointer(xs[k]), pointer(ys[k]), pointer(rs[k]), pointer(cs[k]), pointer(φs[k]),
                       pointer(ψs[k]), size(xs[k], 2), size(ys[k], 2), size(xs[k], 1), 0) for k in 1:K]
    stats = Vector{CBatchStats}(undef, K)
    info = Ref(CBatchInfo())
    cargs = Ref(CArgs(args))
    check(ccall((:culamp_batched_sinkhorn, libculamp), Cint,
                (Ptr{Cvoid}, Ptr{CInstance}, Int32, Ptr{CArgs}, Int64, Float64, UInt32,
                 Ptr{CBatchStats}, Ref{CBatchInfo}, Ptr{Cvoid}),
                handle(), insts, K, cargs, frequency, Float64(p), flags, stats, info, stream_ptr()))
    return φs, ψs, stats
end

"""
    symmetric_sinkhorn(x, marginal, args, frequency=100, p=2; flags=0) -> (f, stats)

Self-transport OT(a, a; x, x) (the symmetric terms of the Sinkhorn divergence)
by the averaged iteration f <- (f + T(f))/2, one row pass per iteration
(culamp_symmetric_sinkhorn); P_ij = exp(f_i + f_j - C_ij / (eta_p W_inf)).
"""
function symmetric_sinkhorn(x::CuArray{Float64}, marginal::CuArray{Float64}, args,
                            frequency::Int=100, p=2; flags::UInt32=UInt32(0))
    d, N = size(x)
    f = CUDA.zeros(Float64, N)
    stats = CStats()
    cargs = Ref(CArgs(args))
    check(ccall((:culamp_symmetric_sinkhorn, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, Int64, Int32, CuPtr{Float64}, Ptr{CArgs}, Int64, Float64,
                 CuPtr{Float64}, UInt32, CuPtr{Float64}, Ref{CStats}, Ptr{CLogRow}, Int64, Ptr{Cvoid}),
                handle(), x, N, d, marginal, cargs, frequency, Float64(p), CU_NULL, flags, f, stats,
                C_NULL, 0, stream_ptr()))
    return f, stats
end

# ---------------------------------------------------------------- gradients

"""
    adjoint_sk(x, y, φ, ψ, eps, p=2) -> grad (d x N)

sum_j P_ij grad_x C(x_i, y_j) for P_ij = exp(φ_i + ψ_j - C_ij / eps) (eps
absolute), one pass over all pairs without storing P (culamp_adjoint_sk). With
solved potentials this is dOT_eps/dx (envelope theorem); dOT/dy is
adjoint_sk(y, x, ψ, φ, eps, p), dOT/da = eps φ, dOT/db = eps ψ.
"""
function adjoint_sk(x::CuArray{Float64}, y::CuArray{Float64}, φ::CuArray{Float64}, ψ::CuArray{Float64},
                    eps::Float64, p=2)
    d, N = size(x)
    M = size(y, 2)
    g = CUDA.zeros(Float64, d, N)
    check(ccall((:culamp_adjoint_sk, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64,
                 Int32, CuPtr{Float64}, CuPtr{Float64}, Float64, Float64, Float64, Ptr{Cvoid}),
                handle(), g, CU_NULL, x, y, N, M, d, φ, ψ, eps, 1.0, Float64(p), stream_ptr()))
    return g
end

# ---------------------------------------------------------------- differentiable OT

"""
    max_cost(x, y, p=2) -> W∞

max_ij C(x_i, y_j) (MirrorProxKernel.jl:280-326 followed by the host maximum),
exact FP64, one launch (culamp_max_cost without row maxima).
"""
function max_cost(x::CuArray{Float64}, y::CuArray{Float64}, p=2)
    d, N = size(x)
    M = size(y, 2)
    w = Ref{Float64}(0.0)
    check(ccall((:culamp_max_cost, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32, Float64,
                 CuPtr{Float64}, Ref{Float64}, Ptr{Cvoid}),
                handle(), x, y, N, M, d, Float64(p), CU_NULL, w, stream_ptr()))
    return w[]
end

# Solver settings of an entropic-OT value solve: eta_p = eps / W∞, stop at L1 <= tol
# (the solvers stop at epsilon / 6), the reference defaults elsewhere
# (src/Utilities.jl:18-31).
_value_args(eta_p, tol) = CArgs(eta_p, 0.0, 1.0, 1.0, 0.01, 1.0, 6.0 * tol, 0.95, 200_000, 10, Inf,
                                Int32(0), Int32(0))

"""
    entropic_ot(x, y, a, b, eps; p=2, tol=1e-7) -> (value, φ, ψ)

OT_eps(a, b; x, y) = min_P <P, C> + eps sum P log P over the couplings of a and b,
by the kernel Sinkhorn at absolute regularisation eps (eta_p = eps / W∞) to L1
marginal error tol; value = eps (a.φ + b.ψ), the dual value at the optimum.
"""
function entropic_ot(x::CuArray{Float64}, y::CuArray{Float64}, a::CuArray{Float64},
                     b::CuArray{Float64}, eps::Float64; p=2, tol::Float64=1e-7)
    d, N = size(x)
    M = size(y, 2)
    winf = max_cost(x, y, p)
    φ = CUDA.zeros(Float64, N)
    ψ = CUDA.zeros(Float64, M)
    stats = CStats()
    cargs = Ref(_value_args(eps / winf, tol))
    check(ccall((:culamp_sinkhorn, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int64, Int64, Int32, CuPtr{Float64},
                 CuPtr{Float64}, Ptr{CArgs}, Int64, Float64, CuPtr{Float64}, CuPtr{Float64}, UInt32,
                 CuPtr{Float64}, CuPtr{Float64}, Ref{CStats}, Ptr{CLogRow}, Int64, Ptr{Cvoid}),
                handle(), x, y, N, M, d, a, b, cargs, 10, Float64(p), CU_NULL, CU_NULL, UInt32(0),
                φ, ψ, stats, C_NULL, 0, stream_ptr()))
    return eps * (dot(a, φ) + dot(b, ψ)), φ, ψ
end

"""
    entropic_ot_self(x, a, eps; p=2, tol=1e-7) -> (value, f)

OT_eps(a, a; x, x) by the symmetric iteration (one potential f = φ = ψ);
value = 2 eps a.f.
"""
function entropic_ot_self(x::CuArray{Float64}, a::CuArray{Float64}, eps::Float64; p=2,
                          tol::Float64=1e-7)
    winf = max_cost(x, x, p)
    args = _value_args(eps / winf, tol)
    d, N = size(x)
    f = CUDA.zeros(Float64, N)
    stats = CStats()
    check(ccall((:culamp_symmetric_sinkhorn, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, Int64, Int32, CuPtr{Float64}, Ptr{CArgs}, Int64, Float64,
                 CuPtr{Float64}, UInt32, CuPtr{Float64}, Ref{CStats}, Ptr{CLogRow}, Int64, Ptr{Cvoid}),
                handle(), x, N, d, a, Ref(args), 10, Float64(p), CU_NULL, UInt32(0), f, stats,
                C_NULL, 0, stream_ptr()))
    return 2 * eps * dot(a, f), f
end

"""
    sinkhorn_divergence(x, y, a, b, eps; p=2, tol=1e-7) -> S

S_eps(a, b; x, y) = OT_eps(a, b) - OT_eps(a, a)/2 - OT_eps(b, b)/2 of the point
clouds x (d x N) and y (d x M) with weights a, b; eps absolute. Differentiable
in x, y, a and b through the rrule below.
"""
sinkhorn_divergence(x, y, a, b, eps; p=2, tol=1e-7) =
    first(_divergence_parts(x, y, a, b, eps, p, tol))

function _divergence_parts(x, y, a, b, eps, p, tol)
    vxy, φ, ψ = entropic_ot(x, y, a, b, Float64(eps); p=p, tol=tol)
    vxx, f = entropic_ot_self(x, a, Float64(eps); p=p, tol=tol)
    vyy, g = entropic_ot_self(y, b, Float64(eps); p=p, tol=tol)
    return vxy - vxx / 2 - vyy / 2, (φ, ψ, f, g)
end

"""
    rrule(::typeof(sinkhorn_divergence), x, y, a, b, eps; p=2, tol=1e-7)

Envelope-theorem gradients at the solved potentials, with eps (and so the
problem) fixed -- W∞ only sets each solve's eta_p = eps / W∞ and does not enter
the value, so it is treated as a constant:
  * dS/dx = adjoint(x, y; φ, ψ) - adjoint(x, x; f, f): x enters both sides of
    OT(a, a), whose plan is symmetric, so its two halves are equal and the
    factor 1/2 cancels; adjoint(x, y; φ, ψ)_i =
    sum_j P_ij grad_x C(x_i, y_j) recomputes P_ij = exp(φ_i + ψ_j - C_ij / eps)
    on the fly (culamp_adjoint_sk) -- nothing N x M is stored;
  * dS/dy symmetrically; dS/da = eps (φ - f), dS/db = eps (ψ - g) (defined up to a
    constant, as sum a = sum b = 1).
eps, p and tol get no tangent.
"""
function ChainRulesCore.rrule(::typeof(sinkhorn_divergence), x::CuArray{Float64},
                              y::CuArray{Float64}, a::CuArray{Float64}, b::CuArray{Float64}, eps;
                              p=2, tol=1e-7)
    S, (φ, ψ, f, g) = _divergence_parts(x, y, a, b, eps, p, tol)
    e = Float64(eps)
    function sinkhorn_divergence_pullback(ΔS)
        Δ = unthunk(ΔS)
        gx = adjoint_sk(x, x, f, f, e, p)
        dx = @thunk(Δ .* (adjoint_sk(x, y, φ, ψ, e, p) .- gx))
        gy = adjoint_sk(y, y, g, g, e, p)
        dy = @thunk(Δ .* (adjoint_sk(y, x, ψ, φ, e, p) .- gy))
        return (NoTangent(), dx, dy, Δ .* e .* (φ .- f), Δ .* e .* (ψ .- g), NoTangent())
    end
    return S, sinkhorn_divergence_pullback
end

"""
    lse_combine!(ψ, parts)

Column potentials of a row-sharded Sinkhorn from the shards' column passes:
ψ_j = -log sum_g exp(-parts[j, g]) (parts: M x G, one column per shard, e.g. an
all-gather of the shards' outputs; culamp_lse_combine).
"""
function lse_combine!(ψ::CuArray{Float64}, parts::CuArray{Float64})
    M, G = size(parts)
    check(ccall((:culamp_lse_combine, libculamp), Cint,
                (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}, Int32, Int64, Ptr{Cvoid}),
                handle(), ψ, parts, G, M, stream_ptr()))
    return ψ
end

end # module
