"""
    LatticeQMCUDA

`multimode=:cuda` for LatticeQM.jl: the k-space routines `bandmatrix`/`getbands`,
`getdensitymatrix!`, `getdos`, `chemicalpotential` and `solvehartreefock` run on one
B200 through `libkspace.so` (C ABI declared in `include/kspace.h`).  No CPU
fallback: a routine that cannot run on the device throws.

Usage:

    using LatticeQM, LatticeQMCUDA
    LatticeQMCUDA.enable!()              # adds :cuda to Parallel.to_executor
    bands = getbands(h, ks; multimode=:cuda)

`enable!` installs the executor; routine-level hooks (a few lines in LatticeQM's `bandmatrix`, `densitymatrix_compute_add!`,
`dos_compute!` and `solveselfconsistent!`) call the `cuda_*` functions below when
the executor is a `CudaExec`.
"""
module LatticeQMCUDA

using LatticeQM
import LatticeQM.Parallel
import LatticeQM.TightBinding: Hops
import LatticeQM.Spectrum
import SparseArrays: SparseMatrixCSC

const LIB = Ref{String}(joinpath(@__DIR__, "..", "lib", "libkspace.so"))

struct CudaExec <: Parallel.Executor
    device::Int
    precision::Symbol   # :fp64 (only :fp64 is built)
end
CudaExec() = CudaExec(0, :fp64)

# ---------------------------------------------------------------- context
mutable struct Context
    ptr::Ptr{Cvoid}
end
const CONTEXTS = Dict{Int,Context}()

function context(device::Int=0)
    get!(CONTEXTS, device) do
        out = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:lqm_ctx_create, LIB[]), Cint, (Cint, Ref{Ptr{Cvoid}}), device, out)
        st == 0 || error("libkspace: cannot create a context on CUDA device $device (status $st)")
        ctx = Context(out[])
        finalizer(c -> ccall((:lqm_ctx_destroy, LIB[]), Cint, (Ptr{Cvoid},), c.ptr), ctx)
        ctx
    end
end

function check(ctx::Context, st::Integer)
    st == 0 && return nothing
    msg = unsafe_string(ccall((:lqm_last_error, LIB[]), Cstring, (Ptr{Cvoid},), ctx.ptr))
    st == -1 ? throw(ArgumentError(msg)) : error("libkspace status $st: $msg")
end

# ---------------------------------------------------------------- k-point shards over GPUs
"""
    comm_unique_id() -> Vector{UInt8}

A communicator id (128 bytes) made on one process and handed to the others (for
example `MPI.Bcast!` or `Distributed.remotecall`), then passed to [`set_comm!`](@ref).
"""
function comm_unique_id()
    id = zeros(UInt8, 128)
    st = ccall((:lqm_comm_unique_id, LIB[]), Cint, (Ptr{UInt8},), id)
    st == 0 || error("libkspace: lqm_comm_unique_id failed (status $st; is libnccl.so.2 loadable?)")
    id
end

"""
    set_comm!(nranks, rank, id; device=0)

Join the k-point shards of `nranks` processes (one GPU each) as `rank` on the
context of `device`.  Afterwards `getdensitymatrix!`, `bandmatrix`, `getdos`,
`chemicalpotential` and `solvehartreefock` with `multimode=:cuda` split the k list
over the ranks (every rank passes the same list) and return the whole-grid result on
every rank, replacing `DistributedExec` (src/modules/Parallel/Parallel.jl:275-287,415-467).
`set_comm!(1, 0, nothing)` removes the communicator.
"""
function set_comm!(nranks::Integer, rank::Integer, id; device::Int=0)
    ctx = context(device)
    if id === nothing
        check(ctx, ccall((:lqm_ctx_set_comm, LIB[]), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{UInt8}),
                         ctx.ptr, nranks, rank, C_NULL))
    else
        length(id) == 128 || throw(ArgumentError("communicator id must be 128 bytes"))
        check(ctx, ccall((:lqm_ctx_set_comm, LIB[]), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{UInt8}),
                         ctx.ptr, nranks, rank, Vector{UInt8}(id)))
    end
    nothing
end

# ---------------------------------------------------------------- Hops upload
mutable struct DeviceHops
    ptr::Ptr{Cvoid}
    ctx::Context
    keys::Vector{Vector{Int}}
end

# Device bytes held by uploaded Hops that no finalizer has released yet.  The
# routines below upload H per call and leave the buffer to the finalizer; past
# LIVE_LIMIT a collection runs first, so that the finalizers of unreachable
# uploads hand their buffers back (to the context's cache) before more are made.
const LIVE_BYTES = Ref{Int}(0)
const LIVE_LIMIT = 4 * 2^30

"""Upload H in its own key order (the Bloch-sum order of `fouriersum!`)."""
function upload(ctx::Context, H)
    ks = collect(keys(H))
    d = length(first(ks))
    n = size(H[first(ks)], 1)
    nbytes = 16 * n * n * length(ks)
    LIVE_BYTES[] + nbytes > LIVE_LIMIT && GC.gc()
    K = Int64[k[i] for i in 1:d, k in ks]                 # d x nR
    out = Ref{Ptr{Cvoid}}(C_NULL)
    if first(values(H)) isa SparseMatrixCSC
        mats = [H[k] for k in ks]
        colptr = [Ptr{Int64}(pointer(m.colptr)) for m in mats]
        rowval = [Ptr{Int64}(pointer(m.rowval)) for m in mats]
        nzval = [Ptr{Float64}(pointer(m.nzval)) for m in mats]
        nnz = Int64[min(length(m.rowval), length(m.nzval)) for m in mats]
        GC.@preserve mats colptr rowval nzval begin
            check(ctx, ccall((:lqm_hops_upload_csc, LIB[]), Cint,
                (Ptr{Cvoid}, Int64, Int64, Int32, Ptr{Int64}, Ptr{Ptr{Int64}}, Ptr{Ptr{Int64}}, Ptr{Ptr{Float64}},
                 Ptr{Int64}, Ref{Ptr{Cvoid}}), ctx.ptr, n, length(ks), d, K, colptr, rowval, nzval, nnz, out))
        end
    else
        B = Array{ComplexF64}(undef, n, n, length(ks))
        for (r, k) in enumerate(ks)
            B[:, :, r] .= H[k]
        end
        check(ctx, ccall((:lqm_hops_upload_dense, LIB[]), Cint,
            (Ptr{Cvoid}, Int64, Int64, Int32, Ptr{Int64}, Ptr{ComplexF64}, Ref{Ptr{Cvoid}}),
            ctx.ptr, n, length(ks), d, K, B, out))
    end
    LIVE_BYTES[] += nbytes
    dh = DeviceHops(out[], ctx, ks)
    finalizer(dh) do h
        LIVE_BYTES[] -= nbytes
        ccall((:lqm_hops_free, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), h.ctx.ptr, h.ptr)
    end
    dh
end

precision_code(e::CudaExec) = e.precision === :fp64 ? Cint(0) :
    throw(ArgumentError("precision=$(e.precision): only :fp64 is built"))

# ---------------------------------------------------------------- routines
"""bands (n x nk) and, with `vectors=true`, U (n x n x nk): `bandmatrix` without projectors."""
function cuda_bandmatrix(H, ks::AbstractMatrix{Float64}, exec::CudaExec; vectors::Bool=false)
    n = size(H[first(keys(H))], 1)
    nk = size(ks, 2)
    if nk == 0  # an empty k-set: the k-loop runs zero times (Spectrum/bands.jl:164-204)
        return vectors ? (zeros(Float64, n, 0), zeros(ComplexF64, n, n, 0)) : zeros(Float64, n, 0)
    end
    ctx = context(exec.device)
    dh = upload(ctx, H)
    bands = zeros(Float64, n, nk)
    U = vectors ? zeros(ComplexF64, n, n, nk) : ComplexF64[]
    check(ctx, ccall((:lqm_bandmatrix, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Ptr{ComplexF64}),
        ctx.ptr, dh.ptr, nk, Matrix{Float64}(ks), vectors, precision_code(exec), bands,
        vectors ? U : Ptr{ComplexF64}(C_NULL)))
    vectors ? (bands, U) : bands
end

"""
    cuda_bandmatrix_obs(H, ks, projectors, exec) -> (bands, obs)

`bandmatrix(H, ks, projectors...)` (Spectrum/bands.jl:164-227) with the band
expectation values obs[i, j, p] = Re ⟨u_i(k_j)| O_p(k_j) |u_i(k_j)⟩
(`lqm_bandmatrix_obs`).  Each projector is an `ExpvalMap` whose operand is a
matrix (k-independent) or a Hops (Bloch-summed at each k); other callables
cannot run on the device and throw.
"""
function cuda_bandmatrix_obs(H, ks::AbstractMatrix{Float64}, projectors, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    n = size(H[first(keys(H))], 1)
    d = length(first(keys(H)))
    dps = DeviceHops[]
    for P in projectors
        op = P isa Spectrum.ExpvalMap ? P.op : P
        if op isa AbstractMatrix
            push!(dps, upload(ctx, Dict(zeros(Int, d) => Matrix{ComplexF64}(op))))
        elseif op isa Hops || op isa AbstractDict
            push!(dps, upload(ctx, op))
        else
            throw(ArgumentError("projector of type $(typeof(op)) cannot run on :cuda (use a matrix or Hops)"))
        end
    end
    nk = size(ks, 2)
    bands = zeros(Float64, n, nk)
    obs = zeros(Float64, n, nk, length(dps))
    ptrs = Ptr{Cvoid}[p.ptr for p in dps]
    GC.@preserve dps begin
        check(ctx, ccall((:lqm_bandmatrix_obs, LIB[]), Cint,
            (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Ptr{Cvoid}}, Ptr{Float64}, Ptr{Float64}),
            ctx.ptr, dh.ptr, nk, Matrix{Float64}(ks), length(dps), ptrs, bands, obs))
    end
    bands, obs
end

"""`density(H, ks, μ)` (Spectrum/dos.jl:20-52) on the device (`lqm_density`)."""
function cuda_density(H, ks::AbstractMatrix{Float64}, μ::Real, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    n = size(H[first(keys(H))], 1)
    out = zeros(Float64, n)
    check(ctx, ccall((:lqm_density, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Float64, Ptr{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Float64(μ), out))
    out
end

"""`ldos(H, ks, frequencies; Γ)` (Spectrum/dos.jl:56-98) on the device (`lqm_ldos`); the
frequency average counts once per k-point (equal to the reference for one frequency)."""
function cuda_ldos(H, ks::AbstractMatrix{Float64}, ωs::AbstractVector, exec::CudaExec; Γ::Real=0.1)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    n = size(H[first(keys(H))], 1)
    out = zeros(Float64, n)
    check(ctx, ccall((:lqm_ldos, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Float64, Ptr{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), length(ωs), Vector{Float64}(ωs), Float64(Γ), out))
    out
end

"""`fermisurfacedensity_fromdata(bandmatrix(H, ks), energies[, obs]; broadening)`
(Spectrum/fermisurface.jl) on the device (`lqm_fermisurface`): (density (nE x nk),
broadening); `broadening=:auto` uses the reference's automatic width."""
function cuda_fermisurfacedensity(H, ks::AbstractMatrix{Float64}, energies::AbstractVector, exec::CudaExec;
                                  broadening=:auto, obs::Union{Nothing,AbstractMatrix}=nothing)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    out = zeros(Float64, length(energies), size(ks, 2))
    g = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_fermisurface, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Float64, Ptr{Float64}, Ptr{Float64},
         Ref{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), length(energies), Vector{Float64}(energies),
        broadening isa Number ? Float64(broadening) : 0.0,
        obs === nothing ? Ptr{Float64}(C_NULL) : Matrix{Float64}(obs), out, g))
    out, g[]
end

"""`berry(H, NX, NY, bandindices)` (Spectrum/berry.jl:140-155) on the device (`lqm_berry`):
(midkgrid, F) with F the (NX-1) x (NY-1) plaquette phases; `bandindices` are 1-based as in
the reference."""
function cuda_berry(H, NX::Int, NY::Int, bandindices::AbstractVector{<:Integer}, exec::CudaExec)
    NY = NY < 1 ? NX : NY
    ctx = context(exec.device)
    dh = upload(ctx, H)
    b = Int64[i - 1 for i in bandindices]
    F = zeros(Float64, NX - 1, NY - 1)
    check(ctx, ccall((:lqm_berry, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int64, Int64, Ptr{Int64}, Ptr{Float64}),
        ctx.ptr, dh.ptr, NX, NY, length(b), b, F))
    midkgrid = [[x; y] for x = range(0.5 / (NX - 1); stop=1 - 0.5 / (NX - 1), length=NX - 1),
                           y = range(0.5 / (NY - 1); stop=1 - 0.5 / (NY - 1), length=NY - 1)]
    midkgrid, F
end

"""`berryalongpath(H, kpoints)` (Spectrum/berry.jl:170-238) on the device (`lqm_berry_path`):
the n x N abelian plaquette phases along the path."""
function cuda_berryalongpath(H, kpoints::AbstractMatrix{Float64}, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    n = size(H[first(keys(H))], 1)
    out = zeros(Float64, n, size(kpoints, 2))
    check(ctx, ccall((:lqm_berry_path, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}),
                     ctx.ptr, dh.ptr, size(kpoints, 2), Matrix{Float64}(kpoints), out))
    out
end

"""`WilsonSlice1D(statesgrid(H, NX, NY, bands)[1:NX-1, 1:NY-1, :, :], dir)` (Spectrum/berry.jl:312-367)
on the device (`lqm_wilson`): (en (nloops x nb), U (nloops x nb x nb)); `bands` 1-based."""
function cuda_wilson_slices(H, NX::Int, NY::Int, bands::AbstractVector{<:Integer}, dir::Int, exec::CudaExec)
    NY = NY < 1 ? NX : NY
    ctx = context(exec.device)
    dh = upload(ctx, H)
    b = Int64[i - 1 for i in bands]
    nl = dir == 1 ? NX - 1 : NY - 1
    en = zeros(Float64, length(b), nl)
    U = zeros(ComplexF64, length(b), length(b), nl)
    check(ctx, ccall((:lqm_wilson, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int64, Int64, Ptr{Int64}, Cint, Ptr{Float64}, Ptr{ComplexF64}),
        ctx.ptr, dh.ptr, NX, NY, length(b), b, dir, en, U))
    permutedims(en), permutedims(U, (3, 1, 2))
end

"""`WilsonWannier2D(H, NX, NY, bandindices)` (Spectrum/berry.jl:274-301) on the device
(`lqm_wilson_wannier`): (p1, p2); `bands` 1-based."""
function cuda_wilson_wannier2d(H, NX::Int, NY::Int, bands::AbstractVector{<:Integer}, exec::CudaExec)
    NY = NY < 1 ? NX : NY
    ctx = context(exec.device)
    dh = upload(ctx, H)
    b = Int64[i - 1 for i in bands]
    p1, p2 = zeros(Float64, length(b)), zeros(Float64, length(b))
    check(ctx, ccall((:lqm_wilson_wannier, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int64, Int64, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}),
        ctx.ptr, dh.ptr, NX, NY, length(b), b, p1, p2))
    p1, p2
end

"""Autotune the one-CTA eigensolver's block size for H's order on sample k-points
(`lqm_autotune_eigh`); the choice stays on the device's context.  Returns
(best block size, its ms, Dict(block size => ms))."""
function cuda_autotune_eigh(H, ks::AbstractMatrix{Float64}, exec::CudaExec; want_rho::Bool=true)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    best, bms, nc = Ref{Cint}(0), Ref{Float64}(0.0), Ref{Int64}(0)
    cnt, cms = zeros(Cint, 16), zeros(Float64, 16)
    check(ctx, ccall((:lqm_autotune_eigh, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Cint, Ref{Cint}, Ref{Float64}, Int64, Ptr{Cint},
         Ptr{Float64}, Ref{Int64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), want_rho, best, bms, 16, cnt, cms, nc))
    Int(best[]), bms[], Dict(Int(cnt[i]) => cms[i] for i in 1:nc[])
end

"""Reduction of the blocked eigensolver: 1 two-stage (dense -> band -> tridiagonal),
0 one-stage panels, -1 the default (two-stage for bands and density passes)."""
cuda_set_two_stage(mode::Int, exec::CudaExec) =
    check(context(exec.device), ccall((:lqm_ctx_set_two_stage, LIB[]), Cint, (Ptr{Cvoid}, Cint),
                                      context(exec.device).ptr, mode))

"""Set the one-CTA eigensolver's block size for order n (0: the built-in rule)."""
cuda_set_eigh_threads(n::Int, nt::Int, exec::CudaExec) =
    check(context(exec.device), ccall((:lqm_ctx_set_eigh_threads, LIB[]), Cint, (Ptr{Cvoid}, Int64, Cint),
                                      context(exec.device).ptr, n, nt))

"""`Wilson2D(H, NX, NY, bandindices)` (Spectrum/berry.jl:258-268) on the device."""
function cuda_wilson2d(H, NX::Int, NY::Int, bands::AbstractVector{<:Integer}, exec::CudaExec)
    en1, U1 = cuda_wilson_slices(H, NX, NY, bands, 1, exec)
    en2, U2 = cuda_wilson_slices(H, NX, NY, bands, 2, exec)
    en1, U1, en2, U2
end

"""Summed plaquette phases of each band manifold (1-based band index vectors) on one
NX x NY state grid (`lqm_berry_flux`)."""
function cuda_berry_flux(H, NX::Int, NY::Int, sets::AbstractVector, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    ptr = Int64[0; cumsum(length.(sets))]
    cols = Int64[b - 1 for s in sets for b in s]
    out = zeros(Float64, length(sets))
    check(ctx, ccall((:lqm_berry_flux, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int64, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}),
        ctx.ptr, dh.ptr, NX, NY, length(sets), ptr, cols, out))
    out
end

"""`getcherns(H, NX, NY, bands)` (Spectrum/berry.jl:378-382) on the device; `bands` 1-based,
all bands when empty."""
function cuda_getcherns(H, NX::Int, NY::Int, bands::AbstractVector, exec::CudaExec)
    NY = NY < 1 ? NX : NY
    n = size(H[first(keys(H))], 1)
    bs = isempty(bands) ? collect(1:n) : collect(bands)
    cuda_berry_flux(H, NX, NY, [[b] for b in bs], exec)
end

"""`gapcherns(H, NX, NY; gaptol)` (Spectrum/berry.jl:470-487) on the device: the gaps from
the device bands on the statesgrid k-points, their Chern numbers from one state grid."""
function cuda_gapcherns(H, NX::Int, NY::Int, exec::CudaExec; gaptol::Real=1e-6)
    NY = NY < 1 ? NX : NY
    ks = reduce(hcat, vec([[x; y] for x in range(0; stop=1, length=NX), y in range(0; stop=1, length=NY)])) .+ 1.34e-8
    E = cuda_bandmatrix(H, Matrix{Float64}(ks), exec)
    emin, emax = vec(minimum(E; dims=2)), vec(maximum(E; dims=2))
    gaps = [(; n=m, elo=emax[m], ehi=emin[m+1]) for m in 1:size(E, 1)-1 if emin[m+1] - emax[m] > gaptol]
    isempty(gaps) && return @NamedTuple{n::Int, elo::Float64, ehi::Float64, chern::Int}[]
    flux = cuda_berry_flux(H, NX, NY, [collect(1:g.n) for g in gaps], exec)
    [(; g.n, g.elo, g.ehi, chern=round(Int, f)) for (g, f) in zip(gaps, flux)]
end

"""`opticalconductivity(frequencies, H, J1, J2, ks; μ, Γ, T)`
(LinearResponse/opticalconductivity.jl:101-127) on the device (`lqm_opticalconductivity`):
the Kubo correlator χ(ω).  `J1`, `J2` are Hops (e.g. from `getcurrentoperators(lat, H)`)."""
function cuda_opticalconductivity(frequencies::AbstractVector, H, J1, J2, ks::AbstractMatrix{Float64},
                                  exec::CudaExec; μ::Float64=0.0, Γ::Float64=0.025, T::Float64=0.1)
    ctx = context(exec.device)
    dh, d1, d2 = upload(ctx, H), upload(ctx, J1), upload(ctx, J2)
    out = zeros(ComplexF64, length(frequencies))
    check(ctx, ccall((:lqm_opticalconductivity, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Float64,
         Float64, Float64, Ptr{ComplexF64}),
        ctx.ptr, dh.ptr, d1.ptr, d2.ptr, size(ks, 2), Matrix{Float64}(ks), length(frequencies),
        Vector{Float64}(frequencies), μ, Γ, T, out))
    out
end

"""`getdensitymatrix!(ρs, H, ks, kweights, μ; T)` on the device; returns the band energy."""
function cuda_densitymatrix!(ρs::Hops, H, ks::AbstractMatrix{Float64}, kweights::AbstractVector{Float64},
                             μ::Float64, T::Real, exec::CudaExec)
    if size(ks, 2) == 0  # an empty k-set: ρ is zeroed and the k-sum is empty (densitymatrix.jl:17-49)
        for k in keys(ρs)
            ρs[k] .= 0
        end
        return 0.0
    end
    ctx = context(exec.device)
    dh = upload(ctx, H)
    Lk = collect(keys(ρs))
    d = length(first(Lk))
    n = size(H[first(keys(H))], 1)
    L = Int64[k[i] for i in 1:d, k in Lk]
    rho = zeros(ComplexF64, n, n, length(Lk))
    eb = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_densitymatrix, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Int64, Ptr{Int64},
         Ptr{ComplexF64}, Ref{Float64}, Cint),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Vector{Float64}(kweights), μ, Float64(T),
        length(Lk), L, rho, eb, precision_code(exec)))
    for (i, k) in enumerate(Lk)
        ρs[k] .= view(rho, :, :, i)
    end
    eb[]
end

"""`getdensitymatrix!(ρ::BdGOperator, H::BdGOperator, ks, kweights, μ; T)`
(Superconductivity/green.jl:38-54) on the device (`lqm_bdg_densitymatrix`): `ρB` and `HB`
are the Nambu Hops (`ρ.h`, `H.h`); returns ⟨H − μN⟩.  `HB` is not modified."""
function cuda_bdg_densitymatrix!(ρB::Hops, HB, ks::AbstractMatrix{Float64}, kweights::AbstractVector{Float64},
                                 μ::Real, T::Real, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, HB)
    Lk = collect(keys(ρB))
    d = length(first(Lk))
    n = size(HB[first(keys(HB))], 1)
    L = Int64[k[i] for i in 1:d, k in Lk]
    rho = zeros(ComplexF64, n, n, length(Lk))
    e = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_bdg_densitymatrix, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Int64, Ptr{Int64},
         Ptr{ComplexF64}, Ref{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Vector{Float64}(kweights), Float64(μ), Float64(T),
        length(Lk), L, rho, e))
    for (i, k) in enumerate(Lk)
        ρB[k] .= view(rho, :, :, i)
    end
    e[]
end

"""`Spectrum.filling(H::BdGOperator, ks, μ; T)` (Superconductivity/operators.jl:117-122) on
the device (`lqm_bdg_filling`); `HB = H.h`."""
function cuda_bdg_filling(HB, ks::AbstractMatrix{Float64}, μ::Real, exec::CudaExec; T::Real=0.01)
    ctx = context(exec.device)
    dh = upload(ctx, HB)
    out = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_bdg_filling, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Ref{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Ptr{Float64}(C_NULL), Float64(μ), Float64(T), out))
    out[]
end

"""`Spectrum.chemicalpotential(H::BdGOperator, ks, target; T, μ_lo, μ_hi)`
(Superconductivity/operators.jl:139-155) on the device (`lqm_bdg_chemicalpotential`)."""
function cuda_bdg_chemicalpotential(HB, ks::AbstractMatrix{Float64}, target::Real, exec::CudaExec;
                                    T::Real=0.01, μ_lo::Real=-100.0, μ_hi::Real=100.0)
    ctx = context(exec.device)
    dh = upload(ctx, HB)
    out = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_bdg_chemicalpotential, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Float64, Float64, Ref{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Ptr{Float64}(C_NULL), Float64(target), Float64(T),
        Float64(μ_lo), Float64(μ_hi), out))
    out[]
end

const WHICH_CODE = Dict(:LM => Cint(0), :SR => Cint(1), :LR => Cint(2))

"""`bandmatrix(H, ks; format=:sparse, num_bands, sigma, which)` on the device
(`lqm_bandmatrix_partial`): per k the `num_bands` eigenpairs of `eigen_sparse`
(Eigen/eigen_sparse_krylovkit.jl:44-88), ascending."""
function cuda_bandmatrix_partial(H, ks::AbstractMatrix{Float64}, num_bands::Int, exec::CudaExec;
                                 sigma::Float64=1e-8, which::Symbol=:LM, vectors::Bool=false)
    n = size(H[first(keys(H))], 1)
    nk = size(ks, 2)
    if nk == 0
        return vectors ? (zeros(Float64, num_bands, 0), zeros(ComplexF64, n, num_bands, 0)) :
               zeros(Float64, num_bands, 0)
    end
    ctx = context(exec.device)
    dh = upload(ctx, H)
    bands = zeros(Float64, num_bands, nk)
    U = vectors ? zeros(ComplexF64, n, num_bands, nk) : ComplexF64[]
    check(ctx, ccall((:lqm_bandmatrix_partial, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Float64, Cint, Cint, Ptr{Float64}, Ptr{ComplexF64}),
        ctx.ptr, dh.ptr, nk, Matrix{Float64}(ks), num_bands, sigma, WHICH_CODE[which], vectors, bands,
        vectors ? U : Ptr{ComplexF64}(C_NULL)))
    vectors ? (bands, U) : bands
end

"""`getdensitymatrix!(ρs, H, ks, kweights, μ; T, format=:sparse, num_bands)` on the device
(`lqm_densitymatrix_partial`): ρ from the selected states only; returns the band energy."""
function cuda_densitymatrix_partial!(ρs::Hops, H, ks::AbstractMatrix{Float64}, kweights::AbstractVector{Float64},
                                     μ::Float64, T::Real, num_bands::Int, exec::CudaExec;
                                     sigma::Float64=1e-8, which::Symbol=:LM)
    if size(ks, 2) == 0
        for k in keys(ρs)
            ρs[k] .= 0
        end
        return 0.0
    end
    ctx = context(exec.device)
    dh = upload(ctx, H)
    Lk = collect(keys(ρs))
    d = length(first(Lk))
    n = size(H[first(keys(H))], 1)
    L = Int64[k[i] for i in 1:d, k in Lk]
    rho = zeros(ComplexF64, n, n, length(Lk))
    eb = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_densitymatrix_partial, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Int64, Float64, Cint, Int64,
         Ptr{Int64}, Ptr{ComplexF64}, Ref{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Vector{Float64}(kweights), μ, Float64(T), num_bands,
        sigma, WHICH_CODE[which], length(Lk), L, rho, eb))
    for (i, k) in enumerate(Lk)
        ρs[k] .= view(rho, :, :, i)
    end
    eb[]
end

"""`chemicalpotential(H, ks, filling; T)` from device bands (unweighted mean, as the reference)."""
function cuda_chemicalpotential(H, ks::AbstractMatrix{Float64}, filling::Real, exec::CudaExec; T::Real=0.0)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    μ = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_chemicalpotential, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Ref{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Ptr{Float64}(C_NULL), Float64(filling),
        Float64(T), μ))
    μ[]
end

"""`dos_compute!` on the device: DOS(ω) = Σ_k w_k Σ_n Im[1/(ω - iΓ - ε)] (/nk when unweighted)."""
function cuda_dos!(DOS::AbstractVector, h, ωs::AbstractVector, ks::AbstractMatrix{Float64}, exec::CudaExec;
                   Γ::Real, kweights=nothing)
    ctx = context(exec.device)
    dh = upload(ctx, h)
    out = zeros(Float64, length(ωs))
    w = kweights === nothing ? Ptr{Float64}(C_NULL) : Vector{Float64}(kweights)
    check(ctx, ccall((:lqm_dos, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Float64}, Float64, Ptr{Float64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), w, length(ωs), Vector{Float64}(ωs), Float64(Γ), out))
    DOS .= out
end

const LOG_CB = Ref{Any}(nothing)
function _log_trampoline(it::Int64, E::Float64, res::Float64, ekin::Float64, eband::Float64, eH::Float64,
                         eF::Float64, μ::Float64, user::Ptr{Cvoid})::Cint
    cb = LOG_CB[]
    cb === nothing && return Cint(0)
    info = (ϵkin=ekin, ϵband=eband, ϵH=eH, ϵF=eF, μ=μ)
    applicable(cb, it, E, res, info) ? cb(it, E, res, info) : cb(it, E, res)
    Cint(0)
end

"""Install `HartreeFock(h, v; hartree, fock, exchange)`'s terms on the context
(`lqm_ctx_set_scf_terms`, `lqm_ctx_set_scf_exchange`; `exchange` an `ExchangeKernel` or
`nothing`)."""
function set_functional!(ctx::Context, hartree::Bool, fock::Bool, exchange)
    check(ctx, ccall((:lqm_ctx_set_scf_terms, LIB[]), Cint, (Ptr{Cvoid}, Cint, Cint), ctx.ptr, hartree, fock))
    if exchange === nothing
        check(ctx, ccall((:lqm_ctx_set_scf_exchange, LIB[]), Cint,
            (Ptr{Cvoid}, Int64, Int64, Int32, Ptr{Int64}, Ptr{ComplexF64}, Int64, Ptr{Int64}, Ptr{Int64}),
            ctx.ptr, 0, 0, 0, C_NULL, C_NULL, 0, C_NULL, C_NULL))
        return nothing
    end
    jk = collect(keys(exchange.j))
    d = length(first(jk))
    ns, nf = size(exchange.sf2idx)
    K = Int64[k[i] for i in 1:d, k in jk]
    B = Array{ComplexF64}(undef, ns, ns, length(jk))
    for (r, k) in enumerate(jk)
        B[:, :, r] .= exchange.j[k]
    end
    siteof = zeros(Int64, ns * nf)
    flavorof = zeros(Int64, ns * nf)
    for a in 1:ns, f in 1:nf
        siteof[exchange.sf2idx[a, f]] = a - 1
        flavorof[exchange.sf2idx[a, f]] = f - 1
    end
    check(ctx, ccall((:lqm_ctx_set_scf_exchange, LIB[]), Cint,
        (Ptr{Cvoid}, Int64, Int64, Int32, Ptr{Int64}, Ptr{ComplexF64}, Int64, Ptr{Int64}, Ptr{Int64}),
        ctx.ptr, ns, length(jk), d, K, B, ns * nf, siteof, flavorof))
    nothing
end

"""Device-resident `solvehartreefock` (linear mixing or Anderson acceleration; density or
commutator residual); returns (ρ, ϵ_GS, info, converged, residual)."""
function cuda_solvehartreefock(h, v, ρ_init::Hops, filling::Real, ks::AbstractMatrix{Float64}, exec::CudaExec;
                               T::Real=0.0, β::Real=1.0, tol::Real=1e-7, iterations::Int=500,
                               log_callback=nothing, acceleration::Symbol=:linear, anderson_depth::Int=5,
                               residual_norm::Symbol=:density, hartree::Bool=true, fock::Bool=true,
                               exchange=nothing, convergenceerror::Bool=false)
    ctx = context(exec.device)
    set_functional!(ctx, hartree, fock, exchange)
    acceleration in (:linear, :anderson) ||
        throw(ArgumentError("acceleration must be :linear or :anderson, got $(acceleration)"))
    residual_norm in (:density, :commutator) ||
        throw(ArgumentError("residual_norm must be :density or :commutator, got $(residual_norm)"))
    depth = acceleration === :anderson ? anderson_depth : 0
    check(ctx, ccall((:lqm_ctx_set_scf_acceleration, LIB[]), Cint, (Ptr{Cvoid}, Cint), ctx.ptr, depth))
    check(ctx, ccall((:lqm_ctx_set_scf_residual, LIB[]), Cint, (Ptr{Cvoid}, Cint), ctx.ptr,
                     residual_norm === :commutator ? 1 : 0))
    dh = upload(ctx, h)
    dv = upload(ctx, v)
    Lk = collect(keys(ρ_init))
    d = length(first(Lk))
    n = size(h[first(keys(h))], 1)
    L = Int64[k[i] for i in 1:d, k in Lk]
    rho = Array{ComplexF64}(undef, n, n, length(Lk))
    for (i, k) in enumerate(Lk)
        rho[:, :, i] .= ρ_init[k]
    end
    out = zeros(Float64, 9)
    LOG_CB[] = log_callback
    cb = @cfunction(_log_trampoline, Cint, (Int64, Float64, Float64, Float64, Float64, Float64, Float64,
                                             Float64, Ptr{Cvoid}))
    check(ctx, ccall((:lqm_scf_hf, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Float64,
         Float64, Int64, Int64, Ptr{Int64}, Ptr{ComplexF64}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}),
        ctx.ptr, dh.ptr, dv.ptr, size(ks, 2), Matrix{Float64}(ks), Ptr{Float64}(C_NULL), Float64(filling),
        Float64(T), Float64(β), Float64(tol), iterations, length(Lk), L, rho, cb, C_NULL, out))
    LOG_CB[] = nothing
    ρ = Hops(Dict(k => rho[:, :, i] for (i, k) in enumerate(Lk)))
    eJ = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_ctx_scf_exchange_energy, LIB[]), Cint, (Ptr{Cvoid}, Ref{Float64}), ctx.ptr, eJ))
    info = (μ=out[2], ϵH=out[3], ϵF=out[4], ϵJ=eJ[], ϵband=out[5], ϵkin=out[6], iterations=Int(out[9]))
    scf_convergence_check(out, convergenceerror)
    ρ, out[1], info, out[8] != 0, out[7]
end

# Not converged: fixedpoint!'s warning (Meanfield/fixedpoint.jl:189-191) and, with
# convergenceerror, solvehartreefock's error (Meanfield/selfconsistent.jl:315-317).
function scf_convergence_check(out, convergenceerror::Bool)
    if out[8] == 0
        @warn("SCF stopped before reaching the tolerance; residual $(out[7]) after $(Int(out[9])) iterations")
        convergenceerror && error("SCF did not converge (convergenceerror = true)")
    end
    nothing
end

"""Device-resident `solvehartreefock` for `HartreeFockBDG` (Superconductivity/hartreefock.jl:5-159):
`h`, `v` the electron-sector Hops, `ρ_init` the Nambu density matrix Hops (`ρ.h`); linear
mixing or Anderson acceleration, the density or commutator residual, the BdG chemical
potential and density matrix per iteration (`lqm_scf_hf_bdg`).
Returns (ρ (Nambu Hops), ϵ_GS, info, converged, residual)."""
function cuda_solvehartreefock_bdg(h, v, ρ_init::Hops, filling::Real, ks::AbstractMatrix{Float64}, exec::CudaExec;
                                   T::Real=0.0, β::Real=1.0, tol::Real=1e-7, iterations::Int=500,
                                   log_callback=nothing, hartree::Bool=true, fock::Bool=true,
                                   acceleration::Symbol=:linear, anderson_depth::Int=5,
                                   residual_norm::Symbol=:density, convergenceerror::Bool=false)
    ctx = context(exec.device)
    acceleration in (:linear, :anderson) ||
        throw(ArgumentError("acceleration must be :linear or :anderson, got $(acceleration)"))
    residual_norm in (:density, :commutator) ||
        throw(ArgumentError("residual_norm must be :density or :commutator, got $(residual_norm)"))
    check(ctx, ccall((:lqm_ctx_set_scf_acceleration, LIB[]), Cint, (Ptr{Cvoid}, Cint), ctx.ptr,
                     acceleration === :anderson ? anderson_depth : 0))
    check(ctx, ccall((:lqm_ctx_set_scf_residual, LIB[]), Cint, (Ptr{Cvoid}, Cint), ctx.ptr,
                     residual_norm === :commutator ? 1 : 0))
    set_functional!(ctx, hartree, fock, nothing)
    dh = upload(ctx, h)
    dv = upload(ctx, v)
    Lk = collect(keys(ρ_init))
    d = length(first(Lk))
    n2 = size(ρ_init[first(Lk)], 1)
    L = Int64[k[i] for i in 1:d, k in Lk]
    rho = Array{ComplexF64}(undef, n2, n2, length(Lk))
    for (i, k) in enumerate(Lk)
        rho[:, :, i] .= ρ_init[k]
    end
    out = zeros(Float64, 10)
    LOG_CB[] = log_callback
    cb = @cfunction(_log_trampoline, Cint, (Int64, Float64, Float64, Float64, Float64, Float64, Float64,
                                             Float64, Ptr{Cvoid}))
    check(ctx, ccall((:lqm_scf_hf_bdg, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Float64, Float64, Float64, Float64, Int64, Int64,
         Ptr{Int64}, Ptr{ComplexF64}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}),
        ctx.ptr, dh.ptr, dv.ptr, size(ks, 2), Matrix{Float64}(ks), Float64(filling), Float64(T), Float64(β),
        Float64(tol), iterations, length(Lk), L, rho, cb, C_NULL, out))
    LOG_CB[] = nothing
    ρ = Hops(Dict(k => rho[:, :, i] for (i, k) in enumerate(Lk)))
    info = (μ=out[2], ϵH=out[3], ϵF=out[4], ϵP=out[10], ϵband=out[5], ϵkin=out[6], iterations=Int(out[9]))
    scf_convergence_check(out, convergenceerror)
    ρ, out[1], info, out[8] != 0, out[7]
end

"""`commutator_kspace_norm(H, ρ, ks; kweights)` (Meanfield/selfconsistent.jl:130-166) on the
device (`lqm_commutator_norm`)."""
function cuda_commutator_kspace_norm(H, ρ, ks::AbstractMatrix{Float64}, exec::CudaExec;
                                     kweights::Union{Nothing,AbstractVector{Float64}}=nothing)
    ctx = context(exec.device)
    dh, dr = upload(ctx, H), upload(ctx, ρ)
    out = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_commutator_norm, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ref{Float64}),
        ctx.ptr, dh.ptr, dr.ptr, size(ks, 2), Matrix{Float64}(ks),
        kweights === nothing ? Ptr{Float64}(C_NULL) : Vector{Float64}(kweights), out))
    out[]
end

# ---------------------------------------------------------------- derivatives
"""
    cuda_densitymatrix(H, ks, kweights, μ, T, Lkeys, exec) -> Dict(L => ρ_L)

Out-of-place `getdensitymatrix!` (keys `Lkeys`), the differentiable form: the
ChainRulesCore extension (`LatticeQMCUDAChainRulesExt.jl`) gives it an `rrule`
through `cuda_densitymatrix_vjp`.
"""
function cuda_densitymatrix(H, ks::AbstractMatrix{Float64}, kweights::AbstractVector{Float64}, μ::Real, T::Real,
                            Lkeys, exec::CudaExec)
    n = size(H[first(keys(H))], 1)
    ρs = Dict(L => zeros(ComplexF64, n, n) for L in Lkeys)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    Lk = collect(Lkeys)
    d = length(first(Lk))
    L = Int64[k[i] for i in 1:d, k in Lk]
    rho = zeros(ComplexF64, n, n, length(Lk))
    eb = Ref{Float64}(0.0)
    check(ctx, ccall((:lqm_densitymatrix, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Int64, Ptr{Int64},
         Ptr{ComplexF64}, Ref{Float64}, Cint),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Vector{Float64}(kweights), Float64(μ), Float64(T),
        length(Lk), L, rho, eb, precision_code(exec)))
    for (i, k) in enumerate(Lk)
        ρs[k] .= view(rho, :, :, i)
    end
    ρs
end

"""
    cuda_densitymatrix_vjp(Ḡ, H, ks, kweights, μ, T, exec) -> Dict(R => H̄_R)

Reverse-mode derivative of the density matrix at fixed μ and T
(`lqm_densitymatrix_vjp`): from Ḡ_L = ∂Loss/∂ρ_L to H̄_R = ∂Loss/∂H_R, with
dLoss = Re Σ_R ⟨H̄_R, dH_R⟩ for Hermitian-consistent perturbations
(dH_{-R} = dH_R'), the ChainRulesCore convention for complex entries.
"""
function cuda_densitymatrix_vjp(Ḡ, H, ks::AbstractMatrix{Float64}, kweights::AbstractVector{Float64}, μ::Real,
                                T::Real, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    n = size(H[first(keys(H))], 1)
    Lk = collect(keys(Ḡ))
    d = length(first(Lk))
    L = Int64[k[i] for i in 1:d, k in Lk]
    G = Array{ComplexF64}(undef, n, n, length(Lk))
    for (i, k) in enumerate(Lk)
        G[:, :, i] .= Ḡ[k]
    end
    out = zeros(ComplexF64, n, n, length(dh.keys))
    check(ctx, ccall((:lqm_densitymatrix_vjp, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Int64, Ptr{Int64},
         Ptr{ComplexF64}, Ptr{ComplexF64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Vector{Float64}(kweights), Float64(μ), Float64(T),
        length(Lk), L, G, out))
    Dict(R => out[:, :, i] for (i, R) in enumerate(dh.keys))
end

"""Reverse-mode derivative of the bands (`lqm_bands_vjp`): ε̄ (n x nk) -> Dict(R => H̄_R)."""
function cuda_bands_vjp(ε̄::AbstractMatrix{Float64}, H, ks::AbstractMatrix{Float64}, exec::CudaExec)
    ctx = context(exec.device)
    dh = upload(ctx, H)
    n = size(H[first(keys(H))], 1)
    out = zeros(ComplexF64, n, n, length(dh.keys))
    check(ctx, ccall((:lqm_bands_vjp, LIB[]), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{ComplexF64}),
        ctx.ptr, dh.ptr, size(ks, 2), Matrix{Float64}(ks), Matrix{Float64}(ε̄), out))
    Dict(R => out[:, :, i] for (i, R) in enumerate(dh.keys))
end

# ---------------------------------------------------------------- executor hooks
# Per-k closures cannot run on the device: the generic k-loops refuse CudaExec.
Parallel.kspace_foreach!(body!, ks::AbstractMatrix, exec::CudaExec; kwargs...) =
    throw(ArgumentError("routine not ported to :cuda"))
Parallel.kspace_reduce!(body!, output, ks::AbstractMatrix, exec::CudaExec; kwargs...) =
    throw(ArgumentError("routine not ported to :cuda"))
Parallel.configure_blas!(::CudaExec; kwargs...) = nothing

"""
    enable!()

Adds `:cuda` to `Parallel.to_executor(::Symbol)` (src/modules/Parallel/Parallel.jl:87-109).
Must run at runtime (Julia does not allow overwriting a method of another
module during precompilation); the other symbols keep their behaviour.
"""
function enable!()
    @eval Parallel function to_executor(s::Symbol)
        if s === :cuda
            $(CudaExec)()
        elseif s === :serial
            SerialExec()
        elseif s === :multithreaded || s === :threaded
            Threads.nthreads() > 1 ? ThreadedExec() : SerialExec()
        elseif s === :distributed
            if nworkers() > 1
                DistributedExec()
            elseif Threads.nthreads() > 1
                ThreadedExec()
            else
                SerialExec()
            end
        elseif s === :auto
            auto()
        else
            @warn "Unknown executor symbol $s; falling back to :serial"
            SerialExec()
        end
    end
    nothing
end

end # module
