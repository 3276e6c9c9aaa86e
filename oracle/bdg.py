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


class HartreeFockBDG:
    """Superconductivity/hartreefock.jl:5-159 (HartreeFockBDG): the electron functional of
    HartreeFock on rho_e (Fock -v .* rho_e, Hartree diag(V0 diag rho_e[0])) and the pairing
    field DeltaMF[L] = v[L] .* rhoD[L] (keys h + v + rhoD), with eP = 1/2 sum Re(|rhoD|^2 v);
    hMF = BdGOperator(hMF_e, DeltaMF).  rho is a Nambu Hops of order 2d."""

    def __init__(self, h, v, hartree=True, fock=True):
        from .meanfield import HartreeFock
        self.hf = HartreeFock(h, v, hartree=hartree, fock=fock)
        self.h, self.v, self.fock = h, v, fock
        self.mu = 0.0
        self.eH = self.eF = self.eP = self.eband = self.ekin = 0.0
        self.hMF_e = None
        self.DMF = None

    def __call__(self, rho):
        d = next(iter(self.h.values())).shape[0]
        rho_e = {L: M[:d, :d] for L, M in rho.items()}
        rhoD = {L: M[:d, d:] for L, M in rho.items()}
        self.hf(rho_e)
        self.hMF_e = self.hf.hMF
        keys = list(self.h.keys()) + [L for L in list(self.v.keys()) + list(rhoD.keys()) if L not in self.h]
        seen, ordered = set(), []
        for L in keys:
            if L not in seen:
                seen.add(L)
                ordered.append(L)
        self.DMF = {L: np.zeros((d, d), complex) for L in ordered}
        if self.fock:
            for L, vL in self.v.items():
                if L in rhoD:
                    self.DMF[L] = self.DMF[L] + vL * rhoD[L]
        self.eH, self.eF = self.hf.eH, self.hf.eF
        self.eP = float(np.real(0.5 * sum(np.sum(rhoD[L] * np.conj(rhoD[L]) * vL)
                                          for L, vL in self.v.items() if L in rhoD))) if self.fock else 0.0
        return self

    def hMF(self):
        return bdg_operator(self.hMF_e, self.DMF)

    def doublecounting(self):
        return self.eH + self.eF + self.eP


def solvehartreefock_bdg(h, v, rho_init, filling, ks, T=0.0, beta=1.0, tol=1e-7, iterations=500,
                         hartree=True, fock=True, log=None, acceleration="linear", anderson_depth=5,
                         residual_norm="density"):
    """solvehartreefock with a Nambu h (Meanfield/selfconsistent.jl:256-336 with the BdG
    methods of Superconductivity: mu from chemicalpotential(::BdGOperator), rho and the band
    energy from getdensitymatrix!(::BdGOperator)); linear mixing (fixedpoint.jl:143-161), or
    Anderson acceleration with the Hermitian projection of the Nambu iterate
    (Superconductivity/hartreefock.jl:57-58); the relative or the commutator residual.
    h is the electron-sector Hops (HartreeFock(h::BdGOperator, v) keeps copyelectronsector(h))."""
    from .meanfield import (hermitianize, is_hermitian, anderson_update, _flatten, _unflatten,
                            commutator_kspace_norm)
    use_anderson = acceleration == "anderson" and anderson_depth > 0
    hist_x, hist_f = [], []
    rho0 = {L: M.copy() for L, M in rho_init.items()}
    if not is_hermitian(rho0):
        hermitianize(rho0)
    rho1 = {L: M.copy() for L, M in rho0.items()}
    hf = HartreeFockBDG(h, v, hartree=hartree, fock=fock)
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk)
    converged, residual, it, E = False, np.inf, 0, 0.0
    while it < iterations:
        it += 1
        hf(rho0)
        HB = hf.hMF()
        comm = commutator_kspace_norm(HB, rho0, ks) if residual_norm == "commutator" else None
        hf.mu = bdg_chemicalpotential(HB, ks, filling, T)
        rho_new, eband = bdg_densitymatrix(HB, ks, w, hf.mu, T, list(rho1.keys()))
        hf.eband = eband
        hf.ekin = eband - 2 * hf.doublecounting()
        E = eband - hf.doublecounting()
        if use_anderson:
            keys = sorted(rho0.keys())
            fx, ff = _flatten(rho0, keys), _flatten(rho_new, keys)
            hist_x.append(fx.copy())
            hist_f.append(ff.copy())
            while len(hist_x) > anderson_depth + 1:
                hist_x.pop(0)
                hist_f.pop(0)
            _unflatten(rho1, anderson_update(fx, ff, hist_x, hist_f, beta), keys)
            hermitianize(rho1)
        else:
            for L in rho0:
                rho1[L] = beta * rho_new[L] + (1 - beta) * rho0[L]
        diff = np.linalg.norm([np.linalg.norm(rho1[L] - rho0[L]) for L in rho0])
        nrm = np.linalg.norm([np.linalg.norm(rho1[L]) for L in rho0])
        residual = diff / nrm if nrm > np.finfo(float).eps else diff
        if comm is not None:
            residual = comm
        for L in rho0:
            rho0[L] = rho1[L].copy()
        if log is not None:
            log(it, E, residual, hf.ekin, hf.eband, hf.eH, hf.eF, hf.mu)
        if residual < tol:
            converged = True
            break
    hf(rho1)
    hf.ekin = hf.eband - 2 * hf.doublecounting()
    E = hf.eband - hf.doublecounting()
    return rho1, E, hf, converged, residual, it
