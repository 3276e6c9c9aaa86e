"""
ChainRulesCore rules for the differentiable device routines of LatticeQMCUDA.

Load after `using ChainRulesCore, LatticeQMCUDA` (as a package extension with
ChainRulesCore as a weak dependency, or by `include` of this file).  Tangents of
the Dict-valued inputs/outputs are Dicts keyed like them; complex cotangents use
the ChainRulesCore convention ∂L/∂Re + i ∂L/∂Im, which is the `Gbar`/`Hbar`
convention of `lqm_densitymatrix_vjp` and `lqm_bands_vjp`.  The hopping
cotangent is exact for Hermitian-consistent parameterisations (H_{-R} = H_R'),
which is how LatticeQM builds Hops.
"""
module LatticeQMCUDAChainRulesExt

using ChainRulesCore
using LatticeQMCUDA: LatticeQMCUDA, CudaExec, cuda_densitymatrix, cuda_densitymatrix_vjp, cuda_bandmatrix,
                     cuda_bands_vjp

function ChainRulesCore.rrule(::typeof(cuda_densitymatrix), H, ks::AbstractMatrix{Float64},
                              kweights::AbstractVector{Float64}, μ::Real, T::Real, Lkeys, exec::CudaExec)
    ρ = cuda_densitymatrix(H, ks, kweights, μ, T, Lkeys, exec)
    function cuda_densitymatrix_pullback(Δρ)
        Ḡ = Dict(L => Matrix{ComplexF64}(unthunk(Δρ)[L]) for L in Lkeys if haskey(unthunk(Δρ), L))
        H̄ = cuda_densitymatrix_vjp(Ḡ, H, ks, kweights, μ, T, exec)
        return (NoTangent(), H̄, NoTangent(), NoTangent(), NoTangent(), NoTangent(), NoTangent(), NoTangent())
    end
    return ρ, cuda_densitymatrix_pullback
end

function ChainRulesCore.rrule(::typeof(cuda_bandmatrix), H, ks::AbstractMatrix{Float64}, exec::CudaExec)
    bands = cuda_bandmatrix(H, ks, exec)
    function cuda_bandmatrix_pullback(Δbands)
        H̄ = cuda_bands_vjp(Matrix{Float64}(unthunk(Δbands)), H, ks, exec)
        return (NoTangent(), H̄, NoTangent(), NoTangent())
    end
    return bands, cuda_bandmatrix_pullback
end

end # module
