"""Nambu (BdG) density matrix, filling and chemical potential restated from LatticeQM.jl
(oracle; test infrastructure only).

A BdG Hamiltonian is a Hops of order 2d (electron block first, then the hole block).
"""
import numpy as np

from . import kspace as K


def bdg_operator(h, delta=None):
    """BdGOperator(h[, Δ]) (Superconductivity/types.jl:43-60,76-97): blocks
    [h_R 0; 0 -conj(h_R)] for R in h, plus [0 Δ_R; Δ_{-R}^H 0] for R in Δ (keys added
    in Δ's order when h lacks them)."""
    d = next(iter(h.values())).shape[0]
    H = {}
    for R, M in h.items():
        B = np.zeros((2 * d, 2 * d), complex)
        B[:d, :d] = M
        B[d:, d:] = -np.conj(M)
        H[R] = B
    if delta:
        for R, D in delta.items():
            mR = tuple(-x for x in R)
            if mR not in delta:
                raise ValueError(f"pairing key {R} has no partner {mR}")
            B = np.zeros((2 * d, 2 * d), complex)
            B[:d, d:] = D
            B[d:, :d] = delta[mR].conj().T
            H[R] = H[R] + B if R in H else B
    return H


def add_chemical_potential(H, mu):
    """addchemicalpotential!(H::BdGOperator, μ) (Superconductivity/operators.jl:14-17) on a
    copy: zero-key electron diagonal + μ, hole diagonal − μ."""
    d = next(iter(H.values())).shape[0] // 2
    z = tuple(0 for _ in next(iter(H.keys())))
    out = {R: M.copy() for R, M in H.items()}
    out[z] = out[z] + np.diag(np.concatenate([np.full(d, mu), np.full(d, -mu)]))
    return out


def bdg_densitymatrix(H, ks, w, mu, T, Lkeys):
    """getdensitymatrix!(ρ::BdGOperator, H::BdGOperator, ks, kweights, μ)
    (Superconductivity/green.jl:38-54): ρ of H shifted by −μ at μ = 0, and the physical
    ⟨H − μN⟩ = (band sum)/2 + (Re tr h_e[0] − d μ)/2."""
    d = next(iter(H.values())).shape[0] // 2
    z = tuple(0 for _ in next(iter(H.keys())))
    rho, eb = K.densitymatrix(add_chemical_potential(H, -mu), ks, w, 0.0, T, Lkeys)
    return rho, eb / 2 + (float(np.real(np.trace(H[z][:d, :d]))) - d * mu) / 2


def bdg_filling(H, ks, mu, T=0.01, w=None):
    """Spectrum.filling(H::BdGOperator, ks, μ; T) (Superconductivity/operators.jl:117-122):
    Re tr ρ_e[0] / d of the BdG density matrix at μ."""
    d = next(iter(H.values())).shape[0] // 2
    z = tuple(0 for _ in next(iter(H.keys())))
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk) if w is None else w
    rho, _ = bdg_densitymatrix(H, ks, w, mu, T, [z])
    return float(np.real(np.trace(rho[z][:d, :d]))) / d


def electron_sector(H):
    d = next(iter(H.values())).shape[0] // 2
    return {R: M[:d, :d].copy() for R, M in H.items()}


def bdg_chemicalpotential(H, ks, filling, T=0.01, w=None, mu_lo=-100.0, mu_hi=100.0):
    """Spectrum.chemicalpotential(H::BdGOperator, ks, target; T) (operators.jl:139-155):
    bracket [max(μ_lo, min ε_e − 1), min(μ_hi, max ε_e + 1)] from the electron-sector
    bands, then Roots' float bisection on filling(μ) − target."""
    bands, _ = K.bandmatrix(electron_sector(H), ks)
    lo = max(mu_lo, float(bands.min()) - 1.0)
    hi = min(mu_hi, float(bands.max()) + 1.0)
    return K.bisect_float(lambda m: bdg_filling(H, ks, m, T, w) - filling, lo, hi)
