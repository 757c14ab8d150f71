"""
    VQCB200

Julia drop-in layer for VQC.jl's state-vector hot path on a B200, over the C
ABI of libvqcb200.so (include/vqc_b200.h).

Status: source only, never executed here — no Julia toolchain exists on the
build image or the GPU boxes.  The same C entry points are exercised by the
Python host mirror (vqc.jl_b200/vqcb200) and the parity tests.

What it provides, method by method (reference file:line in VQC.jl):
  * `CuStateVector` / `CuDensityMatrix`: device-resident StateVector /
    DensityMatrix (statevector.jl:1-21, densitymatrix.jl:1-30);
  * `apply!(::Gate, ::CuStateVector)`, `apply!(::QCircuit, ...)`, `*`
    (applygates/generic/generic.jl:6-33);
  * `expectation(::QubitsOperator|::QubitsTerm, ::CuStateVector)` and the
    two-state form (hamiltonian/expecs/expecs.jl:12-74);
  * ChainRules `rrule`s for `*(::QCircuit, ::CuStateVector)` (circuitdiff.jl:2-8)
    and `expectation(::QubitsOperator, ::CuStateVector)` (expecdiff.jl:68), so
    `Zygote.gradient(c -> real(expectation(h, c * x)), circuit)` runs the
    device adjoint sweep; plus `energy_and_gradient`, the fused form;
  * `partial_tr` and `probabilities` for CuDensityMatrix (ptrace.jl:4-10,
    measure.jl:69-81).
"""
module VQCB200

using LinearAlgebra
using ChainRulesCore
using QuantumCircuits
using QuantumCircuits: ordered_positions, ordered_mat, nparameters, differentiate
import VQC
import VQC: apply!, expectation, partial_tr, storage

export CuStateVector, CuDensityMatrix, energy_and_gradient, probabilities

const libvqc = joinpath(@__DIR__, "..", "vqcb200", "libvqcb200.so")

const VQC_C64 = Cint(0)
const VQC_C128 = Cint(1)
const VQC_PARAM_GENERATOR = Int32(1)

struct VqcGate
    nq::Int32
    pos::NTuple{5,Int32}
    mat::Int64
end

struct VqcParam
    gate::Int32
    kind::Int32
    dmat::Int64
end

struct VqcPauli
    xmask::UInt64
    zmask::UInt64
    coeff_re::Float64
    coeff_im::Float64
end

function check(rc::Integer)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:vqc_last_error, libvqc), Cstring, ()))
    rc == -1 && throw(ArgumentError(msg))
    rc == -4 && throw(msg)              # the reference throws a String (generic.jl:37)
    rc == -2 && throw(OutOfMemoryError())
    error("libvqcb200: " * msg)
end

dtype_code(::Type{ComplexF32}) = VQC_C64
dtype_code(::Type{ComplexF64}) = VQC_C128

# ------------------------------------------------------------------ device states
mutable struct CuStateVector{T<:Union{ComplexF32,ComplexF64}}
    h::Ptr{Cvoid}
    nqubits::Int
    function CuStateVector{T}(n::Int; device::Int=0) where {T}
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:vqc_state_create, libvqc), Cint, (Cint, Cint, Cint, Ptr{Ptr{Cvoid}}),
                    n, dtype_code(T), device, r))
        x = new{T}(r[], n)
        finalizer(x -> ccall((:vqc_state_destroy, libvqc), Cint, (Ptr{Cvoid},), x.h), x)
        return x
    end
end

function CuStateVector(x::VQC.StateVector{T}; device::Int=0) where {T}
    y = CuStateVector{T}(VQC.nqubits(x); device=device)
    v = storage(x)
    check(ccall((:vqc_state_upload, libvqc), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Csize_t),
                y.h, v, sizeof(v)))
    return y
end

function storage(x::CuStateVector{T}) where {T}
    v = Vector{T}(undef, 2^x.nqubits)
    check(ccall((:vqc_state_download, libvqc), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Csize_t), x.h, v, sizeof(v)))
    return v
end

function Base.copy(x::CuStateVector{T}) where {T}
    y = CuStateVector{T}(x.nqubits)
    check(ccall((:vqc_state_copy, libvqc), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), y.h, x.h))
    return y
end

mutable struct CuDensityMatrix{T<:Union{ComplexF32,ComplexF64}}
    h::Ptr{Cvoid}
    nqubits::Int
end

function CuDensityMatrix(x::CuStateVector{T}) where {T}
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:vqc_dm_create, libvqc), Cint, (Cint, Cint, Cint, Ptr{Ptr{Cvoid}}),
                x.nqubits, dtype_code(T), 0, r))
    rho = CuDensityMatrix{T}(r[], x.nqubits)
    finalizer(y -> ccall((:vqc_state_destroy, libvqc), Cint, (Ptr{Cvoid},), y.h), rho)
    check(ccall((:vqc_dm_from_state, libvqc), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), rho.h, x.h))
    return rho
end

# ------------------------------------------------------------------ gates
# ordered_mat is column-major in Julia; the ABI takes row-major, re/im interleaved
rowmajor(m::AbstractMatrix) = reinterpret(Float64, vec(permutedims(ComplexF64.(m))))

function pack_gate(g, mats::Vector{Float64})
    pos = ordered_positions(g)
    p = ntuple(i -> i <= length(pos) ? Int32(pos[i] - 1) : Int32(0), 5)
    off = length(mats)
    append!(mats, rowmajor(ordered_mat(g)))
    return VqcGate(Int32(length(pos)), p, off)
end

function apply!(g::Gate, x::CuStateVector)
    pos = Cint.(collect(ordered_positions(g)) .- 1)
    m = collect(rowmajor(ordered_mat(g)))
    check(ccall((:vqc_apply_gate, libvqc), Cint, (Ptr{Cvoid}, Cint, Ptr{Cint}, Ptr{Float64}),
                x.h, length(pos), pos, m))
    return x
end

function pack_circuit(c::QCircuit; params::Bool=false)
    mats = Float64[]
    gates = VqcGate[]
    ps = VqcParam[]
    for (i, g) in enumerate(c)
        push!(gates, pack_gate(g, mats))
        if params && nparameters(g) > 0
            for G in differentiate(g)       # circuitdiff.jl:29 uses these gates as-is
                off = length(mats)
                append!(mats, rowmajor(ordered_mat(G)))
                push!(ps, VqcParam(Int32(i - 1), VQC_PARAM_GENERATOR, off))
            end
        end
    end
    return gates, mats, ps
end

function apply!(c::QCircuit, x::CuStateVector; fuse::Bool=true)
    gates, mats, _ = pack_circuit(c)
    check(ccall((:vqc_apply_circuit, libvqc), Cint, (Ptr{Cvoid}, Ptr{VqcGate}, Cint, Ptr{Float64}, Cint),
                x.h, gates, length(gates), mats, fuse))
    return x
end

function apply!(c::QCircuit, rho::CuDensityMatrix; fuse::Bool=true)
    gates, mats, _ = pack_circuit(c)
    check(ccall((:vqc_dm_apply_circuit, libvqc), Cint, (Ptr{Cvoid}, Ptr{VqcGate}, Cint, Ptr{Float64}, Cint),
                rho.h, gates, length(gates), mats, fuse))
    return rho
end

Base.:*(c::QCircuit, x::CuStateVector) = apply!(c, copy(x))

# ------------------------------------------------------------------ operators
const PAULIS = ((false, false, ComplexF64[1 0; 0 1]), (true, false, ComplexF64[0 1; 1 0]),
                (true, true, ComplexF64[0 -im; im 0]), (false, true, ComplexF64[1 0; 0 -1]))

"All Pauli strings of a QubitsOperator, identical strings merged."
function pauli_strings(h::QubitsOperator)
    acc = Dict{Tuple{UInt64,UInt64},ComplexF64}()
    for (key, terms) in h.data, (ops, coeff) in terms
        strings = [(UInt64(0), UInt64(0), ComplexF64(coeff))]
        for (q, op) in zip(key, ops)
            next = similar(strings, 0)
            for (x, z, c) in strings, (bx, bz, P) in PAULIS
                a = tr(P * op) / 2
                a == 0 && continue
                push!(next, (x | (UInt64(bx) << (q - 1)), z | (UInt64(bz) << (q - 1)), c * a))
            end
            strings = next
        end
        for (x, z, c) in strings
            acc[(x, z)] = get(acc, (x, z), 0) + c
        end
    end
    return [VqcPauli(x, z, real(c), imag(c)) for ((x, z), c) in acc if c != 0]
end
pauli_strings(t::QubitsTerm) = pauli_strings(QubitsOperator(t))

function expectation(h::Union{QubitsOperator,QubitsTerm}, x::CuStateVector)
    terms = pauli_strings(h)
    out = zeros(Float64, 2)
    check(ccall((:vqc_expect_pauli, libvqc), Cint, (Ptr{Cvoid}, Ptr{VqcPauli}, Cint, Ptr{Float64}),
                x.h, terms, length(terms), out))
    return complex(out[1], out[2])
end

function expectation(y::CuStateVector, h::Union{QubitsOperator,QubitsTerm}, x::CuStateVector)
    terms = pauli_strings(h)
    out = zeros(Float64, 2)
    check(ccall((:vqc_expect_pauli2, libvqc), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{VqcPauli}, Cint, Ptr{Float64}),
                y.h, x.h, terms, length(terms), out))
    return complex(out[1], out[2])
end

function apply_operator(h, x::CuStateVector{T}) where {T}
    terms = pauli_strings(h)
    y = CuStateVector{T}(x.nqubits)
    check(ccall((:vqc_apply_pauli, libvqc), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{VqcPauli}, Cint),
                x.h, y.h, terms, length(terms)))
    return y
end

# ------------------------------------------------------------------ differentiation
"""
    energy_and_gradient(h, circuit, x) -> (E, grads)

E = expectation(h, circuit * x) and d real(E) / d theta for the circuit's
parameters in circuit order, in one device call (forward, Pauli pass,
fused reverse sweep)."""
function energy_and_gradient(h::QubitsOperator, c::QCircuit, x::CuStateVector)
    gates, mats, ps = pack_circuit(c; params=true)
    terms = pauli_strings(h)
    e = zeros(Float64, 2)
    g = zeros(Float64, length(ps))
    check(ccall((:vqc_adjoint_grad, libvqc), Cint,
                (Ptr{Cvoid}, Ptr{VqcGate}, Cint, Ptr{Float64}, Ptr{VqcParam}, Cint, Ptr{VqcPauli}, Cint,
                 Ptr{Float64}, Ptr{Float64}),
                x.h, gates, length(gates), mats, ps, length(ps), terms, length(terms), e, g))
    return complex(e[1], e[2]), g
end

# circuitdiff.jl:2-8: the pullback of circuit * x uncomputes instead of storing
function ChainRulesCore.rrule(::typeof(*), c::QCircuit, x::CuStateVector{T}) where {T}
    y = c * x
    function times_pullback(Δ)
        yy = copy(y)
        Δs = Δ isa CuStateVector ? copy(Δ) : CuStateVector(VQC.StateVector(unthunk(Δ), x.nqubits))
        gates, mats, ps = pack_circuit(c; params=true)
        g = zeros(Float64, length(ps))
        check(ccall((:vqc_circuit_backward, libvqc), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{VqcGate}, Cint, Ptr{Float64}, Ptr{VqcParam}, Cint, Ptr{Float64}),
                    yy.h, Δs.h, gates, length(gates), mats, ps, length(ps), g))
        return NoTangent(), g, Δs
    end
    return y, times_pullback
end

# expecdiff.jl:30-33, 68: pullback (conj(z) h + z h') x
function ChainRulesCore.rrule(::typeof(expectation), h::QubitsOperator, x::CuStateVector)
    E = expectation(h, x)
    function expectation_pullback(z)
        z = unthunk(z)
        Δ = apply_operator(conj(z) * h + z * h', x)
        return NoTangent(), NoTangent(), Δ
    end
    return E, expectation_pullback
end

# ------------------------------------------------------------------ density matrices
function partial_tr(rho::CuDensityMatrix, sites::Vector{Int})
    isempty(sites) && return rho
    m = rho.nqubits - length(sites)
    out = zeros(ComplexF64, 2^m, 2^m)
    s = Cint.(sites .- 1)
    check(ccall((:vqc_dm_ptrace, libvqc), Cint, (Ptr{Cvoid}, Cint, Ptr{Cint}, Ptr{ComplexF64}),
                rho.h, length(s), s, out))
    return out
end

function probabilities(rho::CuDensityMatrix)
    out = zeros(Float64, 2^rho.nqubits)
    check(ccall((:vqc_dm_probs, libvqc), Cint, (Ptr{Cvoid}, Ptr{Float64}), rho.h, out))
    return out
end

end # module
