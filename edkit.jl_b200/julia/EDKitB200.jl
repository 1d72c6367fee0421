"""
    EDKitB200

Julia binding of libedk (include/edk.h): EDKit operators applied on a B200.

    using EDKit, EDKitB200
    B  = TranslationalBasis(L=28, N=14, k=0)
    H  = trans_inv_operator(spin((1.0,"xx"),(1.0,"yy"),(1.0,"zz")), 2, B)
    Hg = B200Operator(H)            # uploads tables and terms once
    y  = Hg * psi                   # H * psi on the GPU
    mul!(y, Hg, psi)                # accumulates, like EDKit's mul!
    E0 = lanczos_e0(Hg, randn(size(Hg,1)); m=300)[1]
    ψt = timeevolve(Hg, ψ0, 0:0.1:10; tol=1e-10)

Not exercised in this repository's tests: Julia is not installed in the build
image; the same entry points are exercised through Python ctypes.
"""
module EDKitB200

using EDKit, LinearAlgebra, SparseArrays
import Base: *, size, eltype
import LinearAlgebra: mul!

export B200Operator, B200Basis, lanczos_e0, ground_state, timeevolve, autotune!, block_lanczos,
       set_search!, KrylovCacheB200, timeevolve!,
       schmidt_b200, ent_S_b200, double_basis_b200, symmetrizer_b200

const libedk = get(ENV, "EDK_LIB", joinpath(@__DIR__, "..", "libedk.so"))

# edk_basis_desc (include/edk.h)
struct BasisDesc
    kind::Int32; L::Int32; base::Int32; a::Int32; k::Int32; p::Int32; N::Int32; ngen::Int32
    gen_order::Ptr{Int32}; gen_q::Ptr{Int32}; gen_perm::Ptr{Int32}; gen_inv::Ptr{UInt8}
    allow::Ptr{UInt64}; D::Int64; I::Ptr{Int64}; R::Ptr{Float64}
end

struct LanczosOpts
    max_steps::Int32; nev::Int32; tol::Float64; check_every::Int32; precision::Int32
    refine_steps::Int32; reorth::Int32; complex_vectors::Int32
end

mutable struct LanczosDiag
    steps::Int32; steps_low::Int32; matvecs::Int32; breakdown::Int32
    seconds::Float64; seconds_matvec::Float64; seconds_reorth::Float64; residual::Float64
    seconds_setup::Float64; seconds_stage1::Float64; seconds_refine::Float64
    refine_rounds::Int32; checks::Int32
    LanczosDiag() = new(0, 0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0)
end

struct KrylovOpts
    tol::Float64; m_init::Int32; m_max::Int32; extend_step::Int32; nsample::Int32
    bisect_iters::Int32; reuse_basis::Int32; extend_basis::Int32; normalize_output::Int32
    precision::Int32
end

mutable struct KrylovDiag
    basis_builds::Int32; basis_extensions::Int32; restarts::Int32; matvecs::Int32
    total_times_served::Int32; max_dim_used::Int32; n_intervals::Int32
    accepted_intervals::NTuple{64, Float64}; seconds::Float64
    KrylovDiag() = new(0, 0, 0, 0, 0, 0, 0, ntuple(_ -> 0.0, 64), 0.0)
end

function check(st)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:edk_last_error, libedk), Cstring, ()))
    error(msg)
end

dtype_code(::Type{Float64}) = Int32(0)
dtype_code(::Type{ComplexF64}) = Int32(1)
dtype_code(::Type{Float32}) = Int32(2)
dtype_code(::Type{ComplexF32}) = Int32(3)

# Basis kind and parameters from the Julia basis object; the tables b.I, b.R
# are passed as EDKit holds them, so the device copy is the same table.
# Symmetry-group bases (AbelianBasis, i.e. every `basis(...)` with k/p/z or
# `symmetries`, and the dedicated Parity/Flip/ParityFlip/TranslationFlip
# types) also pass their generators: order, quantum number, site
# permutation (site i -> perm[i]) and spin-inversion flags, in the order
# AbelianOperator holds them (AbelianBasis.jl:143-193, 771-833).
struct Gens
    order::Vector{Int32}; q::Vector{Int32}; perm::Vector{Int32}; inv::Vector{UInt8}
end
Gens() = Gens(Int32[], Int32[], Int32[], UInt8[])
function push_gen!(G::Gens, order, q, perm, inv)
    push!(G.order, order); push!(G.q, q)
    append!(G.perm, Int32.(perm)); append!(G.inv, UInt8.(inv))
    G
end
# quantum number of a cyclic generator from its phase table c[j] = exp(2πi q j/order)
gen_q(c, order) = order == 1 ? 0 : mod(round(Int, angle(ComplexF64(c[2])) * order / (2π)), order)
# internal momentum K of a translation phase table C[j] = exp(-2πi K j/len)
mom_K(C, len) = length(C) > 1 ? mod(round(Int, -angle(ComplexF64(C[2])) * len / (2π)), len) : 0
reflection(L) = collect(L:-1:1)

function basis_desc(b)
    L = length(b.dgt)
    G = Gens()
    kind, a, k, p = if b isa TensorBasis
        0, 1, 0, 1
    elseif b isa ProjectedBasis
        1, 1, 0, 1
    elseif b isa TranslationalBasis
        len = L ÷ b.A
        2, b.A, mod(-mom_K(b.C, len), len), 1   # the caller's k (the library takes mod(-k, len))
    elseif b isa TranslationParityBasis
        len = L ÷ b.A
        3, b.A, (all(isone, b.C) ? 0 : len ÷ 2), b.P
    elseif b isa AbelianBasis
        Gop = b.G
        for g in eachindex(Gop.g)
            push_gen!(G, Gop.g[g], gen_q(Gop.c[g], Gop.g[g]), Gop.perm[g], Gop.inv[g])
        end
        4, 1, 0, 1
    elseif b isa ParityBasis
        push_gen!(G, 2, b.P == -1 ? 1 : 0, reflection(L), zeros(Bool, L))
        4, 1, 0, 1
    elseif b isa FlipBasis
        push_gen!(G, 2, b.P == -1 ? 1 : 0, collect(1:L), ones(Bool, L))
        4, 1, 0, 1
    elseif b isa ParityFlipBasis
        push_gen!(G, 2, b.P == -1 ? 1 : 0, reflection(L), zeros(Bool, L))
        push_gen!(G, 2, b.Z == -1 ? 1 : 0, collect(1:L), ones(Bool, L))
        4, 1, 0, 1
    elseif b isa TranslationFlipBasis
        len = L ÷ b.A
        perm = [mod(i - b.A - 1, L) + 1 for i in 1:L]   # translation by the unit cell
        push_gen!(G, len, mom_K(b.C, len), perm, zeros(Bool, L))
        push_gen!(G, 2, b.P == -1 ? 1 : 0, collect(1:L), ones(Bool, L))
        5, 1, 0, 1
    else
        error("B200Operator: basis type $(typeof(b)) is not on the GPU path")
    end
    return kind, L, Int32(b.B), a, k, p, G
end

mutable struct B200Basis
    h::Ptr{Cvoid}
    function B200Basis(b)
        kind, L, base, a, k, p, G = basis_desc(b)
        I = kind == 0 ? Int64[] : Vector{Int64}(b.I)
        R = kind <= 1 ? Float64[] : Vector{Float64}(b.R)
        ngen = length(G.order)
        GC.@preserve I R G begin
            d = BasisDesc(kind, L, base, a, k, p, -1, ngen,
                          ngen == 0 ? C_NULL : pointer(G.order), ngen == 0 ? C_NULL : pointer(G.q),
                          ngen == 0 ? C_NULL : pointer(G.perm), ngen == 0 ? C_NULL : pointer(G.inv),
                          C_NULL, length(I), kind == 0 ? C_NULL : pointer(I),
                          kind <= 1 ? C_NULL : pointer(R))
            out = Ref{Ptr{Cvoid}}(C_NULL)
            check(ccall((:edk_basis_create, libedk), Cint, (Ref{BasisDesc}, Ref{Ptr{Cvoid}}), d, out))
        end
        obj = new(out[])
        finalizer(x -> ccall((:edk_basis_destroy, libedk), Cint, (Ptr{Cvoid},), x.h), obj)
        obj
    end
end

"""
    B200Operator(opt::EDKit.Operator)

Upload the merged local terms of `opt` (and its basis tables) to the GPU.
"""
mutable struct B200Operator{Tv}
    h::Ptr{Cvoid}
    basis::B200Basis
    D::Int
    function B200Operator(opt::EDKit.Operator{Tv}) where Tv
        bb = B200Basis(opt.B)
        nsites = Int32[length(s) for s in opt.I]
        sites = Int32.(reduce(vcat, opt.I))
        nnz = Int64[nnz_(m) for m in opt.M]
        colptr = reduce(vcat, [Vector{Int64}(m.colptr) for m in opt.M])
        rowval = reduce(vcat, [Vector{Int64}(m.rowval) for m in opt.M])
        nzval = ComplexF64.(reduce(vcat, [nonzeros(m) for m in opt.M]))
        out = Ref{Ptr{Cvoid}}(C_NULL)
        GC.@preserve nsites sites nnz colptr rowval nzval begin
            check(ccall((:edk_operator_create, libedk), Cint,
                        (Ptr{Cvoid}, Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Int64}, Ptr{Int64},
                         Ptr{Int64}, Ptr{ComplexF64}, Ref{Ptr{Cvoid}}),
                        bb.h, length(opt.M), nsites, sites, nnz, colptr, rowval, nzval, out))
        end
        obj = new{Tv}(out[], bb, size(opt, 1))
        finalizer(x -> ccall((:edk_operator_destroy, libedk), Cint, (Ptr{Cvoid},), x.h), obj)
        obj
    end
end
nnz_(m) = SparseArrays.nnz(m)

size(H::B200Operator) = (H.D, H.D)
size(H::B200Operator, i::Integer) = i <= 2 ? H.D : 1

# mul!(y, H, x): accumulates into y, like EDKit's mul! (Operator.jl:309-328)
function mul!(y::StridedVecOrMat{T}, H::B200Operator, x::StridedVecOrMat{T}) where {T<:Union{Float64,ComplexF64,Float32,ComplexF32}}
    nvec = size(x, 2)
    GC.@preserve x y check(ccall((:edk_apply, libedk), Cint,
        (Ptr{Cvoid}, Int32, Ptr{T}, Ptr{T}, Int64, Int64, Int64, Int32, Int32),
        H.h, dtype_code(T), x, y, nvec, stride(x, 2), stride(y, 2), 1, 0))
    y
end

# H * x: fresh output (Operator.jl:372-394)
function *(H::B200Operator, x::StridedVecOrMat{T}) where {T<:Union{Float64,ComplexF64,Float32,ComplexF32}}
    y = similar(x)
    nvec = size(x, 2)
    GC.@preserve x y check(ccall((:edk_apply, libedk), Cint,
        (Ptr{Cvoid}, Int32, Ptr{T}, Ptr{T}, Int64, Int64, Int64, Int32, Int32),
        H.h, dtype_code(T), x, y, nvec, stride(x, 2), stride(y, 2), 0, 0))
    y
end

"""
    lanczos_e0(H::B200Operator, v0; m=300, nev=1, tol=0.0, precision=:fp64)

Lowest `nev` eigenvalues by Lanczos with full CGS2 reorthogonalisation.
"""
function lanczos_e0(H::B200Operator, v0::AbstractVector{T}; m::Integer=300, nev::Integer=1,
                    tol::Real=0.0, check_every::Integer=10, precision::Symbol=:fp64,
                    refine_steps::Integer=20) where T
    v = Vector{T}(v0)
    o = LanczosOpts(m, nev, tol, check_every, precision === :mixed ? 1 : 0, refine_steps, 1, 0)
    ev = zeros(nev); a = zeros(m); b = zeros(m)
    d = LanczosDiag()
    GC.@preserve v ev a b check(ccall((:edk_lanczos_e0, libedk), Cint,
        (Ptr{Cvoid}, Ref{LanczosOpts}, Ptr{T}, Int32, Int32, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ref{LanczosDiag}), H.h, o, v, dtype_code(T), 0, ev, a, b, d))
    ev, d
end

"""
    ground_state(H::B200Operator, v0; m=300, tol=1e-12, precision=:fp64) -> (E0, ψ, diag)

E0 and the normalised lowest Ritz vector of the same Lanczos run.
"""
function ground_state(H::B200Operator, v0::AbstractVector{T}; m::Integer=300, tol::Real=1e-12,
                      check_every::Integer=10, precision::Symbol=:fp64,
                      refine_steps::Integer=20) where T
    v = Vector{T}(v0)
    o = LanczosOpts(m, 1, tol, check_every, precision === :mixed ? 1 : 0, refine_steps, 1, 0)
    ev = zeros(1)
    Tψ = (T <: Complex || eltype(H) <: Complex) ? ComplexF64 : Float64
    ψ = zeros(Tψ, H.D)
    d = LanczosDiag()
    GC.@preserve v ev ψ check(ccall((:edk_lanczos_ground_state, libedk), Cint,
        (Ptr{Cvoid}, Ref{LanczosOpts}, Ptr{T}, Int32, Int32, Ptr{Float64}, Ptr{Tψ}, Int32,
         Ref{LanczosDiag}), H.h, o, v, dtype_code(T), 0, ev, ψ, dtype_code(Tψ), d))
    ev[1], ψ, d
end
eltype(::B200Operator{Tv}) where Tv = Tv

"""
    timeevolve(H::B200Operator, ψ0, ts; tol=1e-10, m_init=30, m_max=60, ...)

Adaptive Krylov exp(-iHt)ψ0 with EDKit's controller (TimeEvolution.jl:556-649).
"""
function timeevolve(H::B200Operator, ψ0::AbstractVector, ts::AbstractVector{<:Real};
                    tol=1e-10, m_init=30, m_max=60, extend_step=10, nsample=13,
                    bisect_iters=12, reuse_basis=true, extend_basis=true,
                    normalize_output=false, precision::Symbol=:fp64, return_diagnostics=false)
    any(<(0), ts) && error("timeevolve: all times in ts must be non-negative; backward evolution is not supported")
    ψ = Vector{ComplexF64}(ψ0)
    t = Vector{Float64}(ts)
    out = Matrix{ComplexF64}(undef, length(ψ), length(t))
    o = KrylovOpts(tol, m_init, m_max, extend_step, nsample, bisect_iters, reuse_basis,
                   extend_basis, normalize_output, precision === :mixed ? 1 : 0)
    d = KrylovDiag()
    GC.@preserve ψ t out check(ccall((:edk_krylov_evolve, libedk), Cint,
        (Ptr{Cvoid}, Ref{KrylovOpts}, Ptr{ComplexF64}, Ptr{Float64}, Int64, Ptr{ComplexF64},
         Int32, Ref{KrylovDiag}), H.h, o, ψ, t, length(t), out, 0, d))
    return_diagnostics ? (out, d) : out
end
"""
    KrylovCacheB200(H::B200Operator, ψ0; tol=1e-10, m_init=30, m_max=60, ...)

KrylovEvolutionCache on the GPU (TimeEvolution.jl:166-218); advance it with
`timeevolve!(cache, t)` or `timeevolve!(cache, ts)` (forward times only).
"""
mutable struct KrylovCacheB200
    h::Ptr{Cvoid}
    H::B200Operator
    N::Int
    function KrylovCacheB200(H::B200Operator, ψ0::AbstractVector; tol=1e-10, m_init=30,
                             m_max=60, extend_step=10, nsample=13, bisect_iters=12,
                             reuse_basis=true, extend_basis=true, normalize_output=false,
                             precision::Symbol=:fp64)
        ψ = Vector{ComplexF64}(ψ0)
        o = KrylovOpts(tol, m_init, m_max, extend_step, nsample, bisect_iters, reuse_basis,
                       extend_basis, normalize_output, precision === :mixed ? 1 : 0)
        out = Ref{Ptr{Cvoid}}(C_NULL)
        GC.@preserve ψ check(ccall((:edk_krylov_cache_create, libedk), Cint,
            (Ptr{Cvoid}, Ref{KrylovOpts}, Ptr{ComplexF64}, Int32, Ref{Ptr{Cvoid}}),
            H.h, o, ψ, 0, out))
        obj = new(out[], H, length(ψ))
        finalizer(x -> ccall((:edk_krylov_cache_destroy, libedk), Cint, (Ptr{Cvoid},), x.h), obj)
        obj
    end
end

function timeevolve!(c::KrylovCacheB200, ts::AbstractVector{<:Real})
    t = Vector{Float64}(ts)
    out = Matrix{ComplexF64}(undef, c.N, length(t))
    GC.@preserve t out check(ccall((:edk_krylov_cache_evolve, libedk), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{ComplexF64}, Int32), c.h, t, length(t), out, 0))
    out
end
timeevolve!(c::KrylovCacheB200, t::Real) = timeevolve!(c, [t])[:, 1]

# sparse!(opt) / clear_sparse_cache! (Operator.jl:221-285) on the device
function EDKit.sparse!(H::B200Operator)
    n = Ref{Int64}(0)
    check(ccall((:edk_operator_materialize, libedk), Cint, (Ptr{Cvoid}, Int32, Ref{Int64}),
                H.h, 1, n))
    n[]
end
clear_sparse!(H::B200Operator) =
    check(ccall((:edk_operator_materialize, libedk), Cint, (Ptr{Cvoid}, Int32, Ptr{Int64}),
                H.h, 0, C_NULL))

struct TuneResult
    kernel::Int32; search::Int32; tps::Int32; block::Int32; ms::Float64; ncand::Int32
    cand_kernel::NTuple{24, Int32}; cand_search::NTuple{24, Int32}; cand_tps::NTuple{24, Int32}
    cand_block::NTuple{24, Int32}; cand_ms::NTuple{24, Float64}
end

"""
    autotune!(H::B200Operator, T=Float64; nvec=1, materialize=false)

Time every kernel / threads-per-state / index-search choice (and the
materialised matrix with `materialize=true`) on H and keep the fastest.
"""
function autotune!(H::B200Operator, ::Type{T}=Float64; nvec::Integer=1,
                   materialize::Bool=false) where T
    r = Ref{TuneResult}()
    check(ccall((:edk_operator_autotune, libedk), Cint,
                (Ptr{Cvoid}, Int32, Int64, Int32, Ref{TuneResult}),
                H.h, dtype_code(T), nvec, materialize ? 1 : 0, r))
    r[]
end

struct BlockLanczosOpts
    block::Int32; max_steps::Int32; nev::Int32; tol::Float64; check_every::Int32; seed::UInt64
end
mutable struct BlockLanczosDiag
    steps::Int32; matvecs::Int64; breakdowns::Int32; converged::Int32
    seconds::Float64; seconds_spmm::Float64; seconds_orth::Float64; seconds_eig::Float64
    BlockLanczosDiag() = new(0, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
end

"""
    block_lanczos(Hs::Vector{<:B200Operator}; block=64, m=100, nev=4, tol=0.0, seed=1234)

Block Lanczos over all operators at once (e.g. every momentum sector), `block`
seeded random right-hand sides each; returns an nev x length(Hs) matrix of the
lowest distinct eigenvalues.
"""
function block_lanczos(Hs::AbstractVector{<:B200Operator}; block::Integer=64, m::Integer=100,
                       nev::Integer=4, tol::Real=0.0, check_every::Integer=10,
                       seed::Integer=1234)
    hs = Ptr{Cvoid}[H.h for H in Hs]
    o = BlockLanczosOpts(block, m, nev, tol, check_every, seed)
    ev = zeros(nev, length(Hs))
    d = BlockLanczosDiag()
    GC.@preserve hs ev check(ccall((:edk_block_lanczos, libedk), Cint,
        (Int32, Ptr{Ptr{Cvoid}}, Ref{BlockLanczosOpts}, Ptr{Float64}, Ptr{Float64},
         Ref{BlockLanczosDiag}), length(Hs), hs, o, C_NULL, ev, d))
    ev, d
end

timeevolve(H::B200Operator, ψ0::AbstractVector, t::Real; kw...) =
    (t < 0 && error("timeevolve!: requested time $t precedes anchor time 0.0");
     timeevolve(H, ψ0, [t]; kw...)[:, 1])

"""
    set_search!(H::B200Operator, strategy::Symbol)

Index search of the operator's basis: `:hash` (default), `:sorted` (the
binary search of EDKit's `index`) or `:rank` (translation and
translation-parity sectors of fixed N: the rank table, the fastest
matrix-free search).  Rows and results are the same for every choice.
"""
function set_search!(H::B200Operator, strategy::Symbol)
    code = strategy === :hash ? 0 : strategy === :sorted ? 1 : strategy === :rank ? 2 :
           error("unknown index search $strategy")
    check(ccall((:edk_basis_set_search, libedk), Cint, (Ptr{Cvoid}, Int32), H.basis.h, code))
    H
end

# --- eigenvector post-processing (src/Schmidt.jl, src/LinearMap.jl) ---
_vdt(::AbstractVector{Float64}) = Int32(0)
_vdt(::AbstractVector{ComplexF64}) = Int32(1)

"""
    schmidt_b200(v, Ainds, bb::B200Basis, complex_phases::Bool)

EDKit's `schmidt(v, Ainds, b)` (Schmidt.jl:186-336) on the GPU for the basis
uploaded as `bb`; `complex_phases` = `eltype(b) <: Complex`.
"""
function schmidt_b200(v::Vector{T}, Ainds::AbstractVector{<:Integer}, bb::B200Basis,
                      complex_phases::Bool, L::Integer) where {T<:Union{Float64,ComplexF64}}
    a = Int32.(Ainds)
    cm = T <: Complex || complex_phases
    M = zeros(cm ? ComplexF64 : Float64, 2^length(a), 2^(L - length(a)))
    GC.@preserve v a M check(ccall((:edk_schmidt, libedk), Cint,
        (Ptr{Cvoid}, Int32, Ptr{Cvoid}, Int32, Ptr{Int32}, Ptr{Cvoid}, Int32, Int32),
        bb.h, _vdt(v), v, length(a), a, M, cm ? 1 : 0, 0))
    M
end

"""
    ent_S_b200(v, Aind, bb::B200Basis; α=1, cutoff=1e-20)

EDKit's `ent_S` (Schmidt.jl:150-153) with the Schmidt matrix and its spectrum
on the GPU.
"""
function ent_S_b200(v::Vector{T}, Aind::AbstractVector{<:Integer}, bb::B200Basis;
                    α::Real=1, cutoff::Real=1e-20) where {T<:Union{Float64,ComplexF64}}
    a = Int32.(Aind)
    S = Ref{Float64}(0.0)
    GC.@preserve v a check(ccall((:edk_ent_S, libedk), Cint,
        (Ptr{Cvoid}, Int32, Ptr{Cvoid}, Int32, Ptr{Int32}, Float64, Float64, Ref{Float64}, Int32),
        bb.h, _vdt(v), v, length(a), a, α, cutoff, S, 0))
    iszero(α) ? round(Int, S[]) : S[]
end

"""
    double_basis_b200(B1::B200Basis, B2::B200Basis, D1, v)

`(DoubleBasis(B1, B2))(v)` (LinearMap.jl:140-166) on the GPU; returns a
ComplexF64 vector of length `D1 = size(B1, 1)`.
"""
function double_basis_b200(B1::B200Basis, B2::B200Basis, D1::Integer,
                           v::Vector{T}) where {T<:Union{Float64,ComplexF64}}
    out = zeros(ComplexF64, D1)
    GC.@preserve v out check(ccall((:edk_double_basis_apply, libedk), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int32, Ptr{Cvoid}, Ptr{ComplexF64}, Int32),
        B1.h, B2.h, _vdt(v), v, out, 0))
    out
end

"""
    symmetrizer_b200(B1::B200Basis, B2::B200Basis, D1, D2)

`symmetrizer(DoubleBasis(B1, B2))` (LinearMap.jl:183-185) on the GPU.
"""
function symmetrizer_b200(B1::B200Basis, B2::B200Basis, D1::Integer, D2::Integer)
    M = zeros(ComplexF64, D1, D2)
    GC.@preserve M check(ccall((:edk_symmetrizer, libedk), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{ComplexF64}, Int32), B1.h, B2.h, M, 0))
    M
end

end # module
