# PauliOperatorsGPU: GPU-resident SparsePauliVector methods for PauliOperators.jl,
# calling libpauliprop.so (include/pauliprop.h) through ccall.
#
# Mirrors the reference's SparsePauliVector API (src/type_SparsePauliVector.jl,
# src/spv_evolve.jl, src/channels.jl) for real (Float64) coefficients.  Term
# arrays stay on the GPU between calls; Julia owns host arrays only for the
# duration of a call.  Not exercised in this repository (no Julia toolchain where
# it was built); the same C ABI is tested from Python (tests/).
module PauliOperatorsGPU

using PauliOperators
using LinearAlgebra
using Random
using PauliOperators: MergeFilter, NOFILTER, _compile_filter, _is_compilable, _pack, _unpack, _word_type,
                      CorrectionAccumulator, NoCorrection, EnergyCorrection, EnergyVarianceCorrection,
                      AdaptiveTruncation, StochasticCoeffTruncation, StochasticSamplingTruncation,
                      TruncationStrategy, CompositeTruncation

const LIB = get(ENV, "PAULIPROP_LIB", joinpath(@__DIR__, "..", "lib", "libpauliprop.so"))

# pp_filter is byte-identical to the isbits MergeFilter (spv_kernels.jl:33-42).
@assert sizeof(MergeFilter) == 64

struct PPCounters
    nwin::Int64
    terms_created::Ptr{Int64}
    merge_in::Ptr{Int64}
    merge_out::Ptr{Int64}
    early_merges::Ptr{Int64}
    t_rotate::Ptr{Float64}
    t_merge::Ptr{Float64}
end

struct PPEvolveOpts
    window::Int64
    strict::Ptr{MergeFilter}
    local_::Ptr{MergeFilter}
    strict_kind::Int32
    corr_kind::Int32
    adapt_max_terms::Int64
    adapt_min_thresh::Float64
    ket::Ptr{Cvoid}
    corr_energy::Ptr{Float64}
    counters::Ptr{PPCounters}
    chan_kind::Int32
    pad::Int32
    chan_prm::NTuple{3,Float64}
    chan_mask::Ptr{Cvoid}
    expect_out::Ptr{Float64}
    chan_every::Int64
    stats_out::Ptr{Float64}
    profile::Int32
    pad2::Int32
    corr_variance::Ptr{Float64}
    seed::UInt64
end

const ERRORS = Dict(1 => ArgumentError, 2 => DimensionMismatch)

function check(st::Cint)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:pp_last_error, LIB), Cstring, ()))
    st == 1 && throw(ArgumentError(msg))
    st == 2 && throw(DimensionMismatch(msg))
    st == 4 && throw(OutOfMemoryError())
    error(msg)
end

"""
    CuSparsePauliVector{N,W}

GPU-resident counterpart of `SparsePauliVector{N,W,Float64}`.
"""
mutable struct CuSparsePauliVector{N,W<:Unsigned}
    h::Ptr{Cvoid}
    function CuSparsePauliVector{N,W}(live_cap::Int, append_cap::Int) where {N,W}
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:pp_create, LIB), Cint, (Int32, Int64, Int64, Ref{Ptr{Cvoid}}), N, live_cap, append_cap, r))
        v = new{N,W}(r[])
        finalizer(x -> ccall((:pp_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), v)
        return v
    end
    # wrap an existing handle (pp_copy)
    function CuSparsePauliVector{N,W}(h::Ptr{Cvoid}) where {N,W}
        v = new{N,W}(h)
        finalizer(x -> ccall((:pp_destroy, LIB), Cint, (Ptr{Cvoid},), x.h), v)
        return v
    end
end

# SparsePauliVector(O::PauliSum; T=Float64, ...) (type_SparsePauliVector.jl:167-188)
function CuSparsePauliVector(O::PauliSum{N}; capacity_factor::Real=2.0, append_factor::Real=1.0,
                             min_capacity::Int=16, imag_tol::Real=1e-10) where {N}
    v = SparsePauliVector(O; T=Float64, capacity_factor, append_factor, min_capacity, imag_tol)
    return CuSparsePauliVector(v)
end

function CuSparsePauliVector(v::SparsePauliVector{N,W,Float64}) where {N,W}
    g = CuSparsePauliVector{N,W}(length(v.z), length(v.az))
    check(ccall((:pp_upload, LIB), Cint, (Ptr{Cvoid}, Ptr{W}, Ptr{W}, Ptr{Float64}, Int64, Int32),
                g.h, v.z, v.x, v.c, v.n, 1))
    return g
end

Base.length(v::CuSparsePauliVector) = (r = Ref{Int64}(0);
    check(ccall((:pp_length, LIB), Cint, (Ptr{Cvoid}, Ref{Int64}), v.h, r)); Int(r[]))

# PauliSum(v) gather (type_SparsePauliVector.jl:212-221)
function PauliOperators.PauliSum(v::CuSparsePauliVector{N,W}) where {N,W}
    n = length(v)
    z = Vector{W}(undef, n); x = Vector{W}(undef, n); c = Vector{Float64}(undef, n)
    r = Ref{Int64}(0)
    check(ccall((:pp_download, LIB), Cint, (Ptr{Cvoid}, Ptr{W}, Ptr{W}, Ptr{Float64}, Int64, Ref{Int64}),
                v.h, z, x, c, n, r))
    out = PauliSum(N, Float64)
    for i in 1:n
        out[_unpack(PauliBasis{N}, z[i], x[i])] = c[i]
    end
    return out
end

# evolve!(O, G, θ) (spv_evolve.jl:228-236)
function PauliOperators.evolve!(v::CuSparsePauliVector{N,W}, G::PauliBasis{N}, θ::Real) where {N,W}
    gz, gx = _pack(W, G)
    check(ccall((:pp_evolve1, LIB), Cint, (Ptr{Cvoid}, Ref{W}, Ref{W}, Float64, Float64),
                v.h, gz, gx, cos(θ), sin(θ)))
    return v
end

# evolve!(O, generators, angles; window, truncation, local_truncation, correction)
# (spv_evolve.jl:312-387)
function PauliOperators.evolve!(v::CuSparsePauliVector{N,W}, gens::Vector{PauliBasis{N}}, angles::Vector{<:Real};
                                window::Int=1, truncation=NoTruncation(), local_truncation=NoTruncation(),
                                correction::CorrectionAccumulator=NoCorrection()) where {N,W}
    length(gens) == length(angles) || throw(DimensionMismatch("generators and angles must have same length"))
    _is_compilable(local_truncation) ||
        throw(ArgumentError("local_truncation must be a deterministic (weight/coefficient) strategy — it runs per append"))
    gz = Vector{W}(undef, length(gens)); gx = similar(gz)
    for i in eachindex(gens)
        gz[i], gx[i] = _pack(W, gens[i])
    end
    cs = cos.(Float64.(angles)); sn = sin.(Float64.(angles))
    strict = Ref(_is_compilable(truncation) ? _compile_filter(truncation) : NOFILTER)
    loc = Ref(_compile_filter(local_truncation))
    kind, mt, mn, seed = Int32(0), 0, 0.0, UInt64(0)
    if truncation isa AdaptiveTruncation
        kind, mt, mn = Int32(1), truncation.max_terms, truncation.min_thresh
    elseif truncation isa StochasticCoeffTruncation
        kind, mn, seed = Int32(2), truncation.epsilon, rand(truncation.rng, UInt64)
    elseif truncation isa StochasticSamplingTruncation
        kind, mt, seed = Int32(3), truncation.n_keep, rand(truncation.rng, UInt64)
    elseif !_is_compilable(truncation)
        throw(ArgumentError("$(typeof(truncation)) has no GPU path (no CPU fallback)"))
    end
    ket = Ref{W}(zero(W)); ce = Ref(0.0); cv = Ref(0.0); corr = Int32(0)
    if correction isa Union{EnergyCorrection,EnergyVarianceCorrection}
        corr = correction isa EnergyVarianceCorrection ? Int32(2) : Int32(1)
        ket[] = (correction.ψ.v % UInt128) % W; ce[] = correction.accumulated_energy
        correction isa EnergyVarianceCorrection && (cv[] = correction.accumulated_variance)
    end
    GC.@preserve strict loc ket ce cv gz gx cs sn begin
        opts = Ref(PPEvolveOpts(window, Base.unsafe_convert(Ptr{MergeFilter}, strict),
                                Base.unsafe_convert(Ptr{MergeFilter}, loc), kind, corr, mt, mn,
                                Base.unsafe_convert(Ptr{W}, ket), Base.unsafe_convert(Ptr{Float64}, ce),
                                C_NULL, Int32(-1), Int32(0), (0.0, 0.0, 0.0), C_NULL, C_NULL, 0, C_NULL,
                                Int32(0), Int32(0), Base.unsafe_convert(Ptr{Float64}, cv), seed))
        check(ccall((:pp_evolve, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{W}, Ptr{W}, Ptr{Float64}, Ptr{Float64}, Int64, Ref{PPEvolveOpts}),
                    v.h, gz, gx, cs, sn, length(gens), opts))
    end
    correction isa Union{EnergyCorrection,EnergyVarianceCorrection} && (correction.accumulated_energy = ce[])
    correction isa EnergyVarianceCorrection && (correction.accumulated_variance = cv[])
    return v
end

# variance(v, ψ) (statistics.jl:6-22)
function PauliOperators.variance(v::CuSparsePauliVector{N,W}, ψ::Ket{N}) where {N,W}
    k = Ref((ψ.v % UInt128) % W); out = Ref(0.0)
    check(ccall((:pp_variance, LIB), Cint, (Ptr{Cvoid}, Ref{W}, Ref{Float64}), v.h, k, out))
    return out[]
end

# clip family (spv_evolve.jl:13-26) and compilable truncate! (truncation.jl:330-337)
function _compact!(v::CuSparsePauliVector, s)
    f = Ref(_compile_filter(s))
    check(ccall((:pp_compact, LIB), Cint, (Ptr{Cvoid}, Ref{MergeFilter}), v.h, f))
    return v
end
PauliOperators.coeff_clip!(v::CuSparsePauliVector, t::Real) = _compact!(v, CoeffTruncation(Float64(t)))
PauliOperators.weight_clip!(v::CuSparsePauliVector, w::Int) = _compact!(v, WeightTruncation(w))
PauliOperators.x_weight_clip!(v::CuSparsePauliVector, w::Int) = _compact!(v, XWeightTruncation(w))
PauliOperators.majorana_weight_clip!(v::CuSparsePauliVector, w::Int) = _compact!(v, MajoranaWeightTruncation(w))
PauliOperators.weight_damped_clip!(v::CuSparsePauliVector, a::Real, t::Real) =
    _compact!(v, WeightDampedTruncation(Float64(a), Float64(t)))
PauliOperators.x_weight_damped_clip!(v::CuSparsePauliVector, a::Real, t::Real) =
    _compact!(v, XWeightDampedTruncation(Float64(a), Float64(t)))

# _apply!(v, ::AdaptiveTruncation) (spv_evolve.jl:103-114): exact top-k clip on the device
function _adaptive!(v::CuSparsePauliVector, s::AdaptiveTruncation)
    check(ccall((:pp_adaptive, LIB), Cint, (Ptr{Cvoid}, Int64, Float64), v.h, s.max_terms, s.min_thresh))
    return v
end

# truncate!(O, strategy, corr) (truncation.jl:330-337) for the strategies with a device path
function PauliOperators.truncate!(v::CuSparsePauliVector{N}, s::TruncationStrategy,
                                  corr::CorrectionAccumulator=NoCorrection()) where {N}
    before = corr isa EnergyCorrection ? expectation_value(v, corr.ψ) : 0.0
    if s isa AdaptiveTruncation
        _adaptive!(v, s)
    elseif s isa StochasticCoeffTruncation
        check(ccall((:pp_stochastic_clip, LIB), Cint, (Ptr{Cvoid}, Float64, UInt64), v.h, s.epsilon, rand(s.rng, UInt64)))
    elseif s isa StochasticSamplingTruncation
        check(ccall((:pp_stochastic_sample, LIB), Cint, (Ptr{Cvoid}, Int64, UInt64), v.h, s.n_keep, rand(s.rng, UInt64)))
    elseif s isa CompositeTruncation
        foreach(x -> PauliOperators.truncate!(v, x), s.strategies)
    elseif _is_compilable(s)
        _compact!(v, s)
    else
        throw(ArgumentError("$(typeof(s)) has no GPU path (no CPU fallback)"))
    end
    corr isa EnergyCorrection && (corr.accumulated_energy += expectation_value(v, corr.ψ) - before)
    return v
end

# stochastic_clip!(v, ε; rng) (spv_evolve.jl:35-52)
PauliOperators.stochastic_clip!(v::CuSparsePauliVector, ε::Real; rng=Random.default_rng()) =
    (check(ccall((:pp_stochastic_clip, LIB), Cint, (Ptr{Cvoid}, Float64, UInt64), v.h, ε, rand(rng, UInt64))); v)

# channels (channels.jl:203-265)
function _channel!(v::CuSparsePauliVector{N,W}, kind::Integer, prm, qubits) where {N,W}
    M = Ref((PauliOperators._qubit_mask(N, qubits) % UInt128) % W)
    p = Float64[prm...; zeros(3 - length(prm))]
    check(ccall((:pp_channel, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ref{W}), v.h, kind, p, M))
    return v
end
PauliOperators.depolarizing_channel!(v::CuSparsePauliVector, p::Real; qubits=nothing) = _channel!(v, 0, (p,), qubits)
PauliOperators.dephasing_channel!(v::CuSparsePauliVector, p::Real; qubits=nothing) = _channel!(v, 1, (p,), qubits)
PauliOperators.bit_flip_channel!(v::CuSparsePauliVector, p::Real; qubits=nothing) = _channel!(v, 2, (p,), qubits)
PauliOperators.bit_phase_flip_channel!(v::CuSparsePauliVector, p::Real; qubits=nothing) = _channel!(v, 3, (p,), qubits)
PauliOperators.pauli_channel!(v::CuSparsePauliVector, pX::Real, pY::Real, pZ::Real; qubits=nothing) =
    _channel!(v, 4, (pX, pY, pZ), qubits)

# expectation_value(v, ::Ket) (spv_evolve.jl:133-134)
function PauliOperators.expectation_value(v::CuSparsePauliVector{N,W}, ψ::Ket{N}) where {N,W}
    k = Ref((ψ.v % UInt128) % W); out = Ref(0.0)
    check(ccall((:pp_expect_ket, LIB), Cint, (Ptr{Cvoid}, Ref{W}, Ref{Float64}), v.h, k, out))
    return out[]
end

# check_spv (type_SparsePauliVector.jl:263-278)
function check_spv(v::CuSparsePauliVector)
    ok = Ref{Int32}(0)
    check(ccall((:pp_check, LIB), Cint, (Ptr{Cvoid}, Ref{Int32}), v.h, ok))
    ok[] == 1 || error("live keys not strictly increasing")
    return true
end

# SparsePauliVector algebra (spv_ops.jl), real coefficients
function Base.copy(v::CuSparsePauliVector{N,W}) where {N,W}
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:pp_copy, LIB), Cint, (Ptr{Cvoid}, Ref{Ptr{Cvoid}}), v.h, r))
    o = CuSparsePauliVector{N,W}(r[])
    return o
end
LinearAlgebra.mul!(v::CuSparsePauliVector, a::Real) =
    (check(ccall((:pp_scale, LIB), Cint, (Ptr{Cvoid}, Float64), v.h, a)); v)
Base.:*(v::CuSparsePauliVector, a::Real) = mul!(copy(v), a)
Base.:*(a::Real, v::CuSparsePauliVector) = v * a
Base.:-(v::CuSparsePauliVector) = v * -1
function LinearAlgebra.norm(v::CuSparsePauliVector, p::Real=2)
    out = Ref(0.0)
    check(ccall((:pp_norm, LIB), Cint, (Ptr{Cvoid}, Float64, Ref{Float64}), v.h, p, out))
    return out[]
end
function LinearAlgebra.tr(v::CuSparsePauliVector)
    out = Ref(0.0)
    check(ccall((:pp_trace, LIB), Cint, (Ptr{Cvoid}, Ref{Float64}), v.h, out))
    return out[]
end
Base.sum!(v1::CuSparsePauliVector{N}, v2::CuSparsePauliVector{N}) where {N} =
    (check(ccall((:pp_sum, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Float64), v1.h, v2.h, 1.0)); v1)
Base.:+(v1::CuSparsePauliVector{N}, v2::CuSparsePauliVector{N}) where {N} = sum!(copy(v1), v2)
Base.:-(v1::CuSparsePauliVector{N}, v2::CuSparsePauliVector{N}) where {N} =
    (o = copy(v1); check(ccall((:pp_sum, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Float64), o.h, v2.h, -1.0)); o)
function PauliOperators.inner_product(v1::CuSparsePauliVector{N}, v2::CuSparsePauliVector{N}) where {N}
    out = Ref(0.0)
    check(ccall((:pp_inner_product, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Float64}), v1.h, v2.h, out))
    return out[]
end
_product!(out::CuSparsePauliVector, A::CuSparsePauliVector, B::CuSparsePauliVector, kind) =
    (check(ccall((:pp_product, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int32), out.h, A.h, B.h, kind)); out)
Base.:*(A::CuSparsePauliVector{N,W}, B::CuSparsePauliVector{N,W}) where {N,W} =
    _product!(CuSparsePauliVector{N,W}(16, 16), A, B, 0)
PauliOperators.anticommutator!(out::CuSparsePauliVector, A::CuSparsePauliVector, B::CuSparsePauliVector) =
    _product!(out, A, B, 1)
PauliOperators.commutator!(out::CuSparsePauliVector, A::CuSparsePauliVector, B::CuSparsePauliVector) =
    _product!(out, A, B, 2)

export CuSparsePauliVector, check_spv

end # module
