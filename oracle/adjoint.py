"""Oracle for the reverse-mode derivatives of the k-space path (TEST INFRASTRUCTURE).

The reference has no derivatives; these are the analytic adjoints of its forward
maps, restated in NumPy and pinned against central finite differences of the
forward oracle (``tests/test_oracle_pins.py``):

* density response of ``getdensitymatrix!`` (Operators/densitymatrix.jl:17-49,
  130-145) at fixed mu and T: for a Hermitian dH(k),
  d rho_k = U [F o (U^H dH(k) U)] U^H with F_ij = (f_i - f_j)/(eps_i - eps_j)
  (the derivative f'((eps_i + eps_j)/2) when |eps_i - eps_j| <= 1e-6 T, and 0
  for equal eigenvalues at T = 0);
* bands of ``bandmatrix`` (Spectrum/bands.jl:164-227): d eps_j = u_j^H dH(k) u_j.

Convention: dLoss = Re sum_L <Gbar_L, d rho_L> = Re sum_R <Hbar_R, dH_R>, where
<A, B> = sum conj(A) B, for Hermitian-consistent perturbations dH_{-R} = dH_R^H.
"""
import math

import numpy as np

from . import kspace as K


def _phase(k, R, sign):
    return np.exp(sign * 1j * 2 * math.pi * float(np.dot(k, np.array(R, float))))


def fermi_matrix(eps, mu, T):
    """F_ij of the density response (divided difference of the Fermi function)."""
    eps = np.asarray(eps, float)
    f = K.fermidirac(eps, mu, T)
    d = eps[:, None] - eps[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        F = (f[:, None] - f[None, :]) / d
    if T > 0:
        mid = 0.5 * (eps[:, None] + eps[None, :])
        fm = K.fermidirac(mid, mu, T)
        slope = -fm * (1.0 - fm) / T
        F = np.where(np.abs(d) <= 1e-6 * T, slope, F)
    else:
        F = np.where(d == 0.0, 0.0, F)
    return F


def densitymatrix_vjp(h, ks, w, mu, T, Gbar):
    """Hbar_R = sum_k e^{-i2pi k.R} w_k U [F o (U^H B_k U)] U^H, B_k = sum_L e^{+i2pi k.L} Gbar_L."""
    n = next(iter(h.values())).shape[0]
    out = {R: np.zeros((n, n), complex) for R in h}
    for j in range(ks.shape[1]):
        k = ks[:, j]
        eps, U = K.eigh_upper(K.fouriersum(h, k))
        Bk = sum(_phase(k, L, +1) * G for L, G in Gbar.items())
        X = U.conj().T @ Bk @ U
        Hk = w[j] * (U @ (fermi_matrix(eps, mu, T) * X) @ U.conj().T)
        for R in h:
            out[R] += _phase(k, R, -1) * Hk
    return out


def bands_vjp(h, ks, eps_bar):
    """Hbar_R = sum_k e^{-i2pi k.R} U diag(eps_bar_k) U^H."""
    n = next(iter(h.values())).shape[0]
    out = {R: np.zeros((n, n), complex) for R in h}
    for j in range(ks.shape[1]):
        k = ks[:, j]
        _, U = K.eigh_upper(K.fouriersum(h, k))
        Hk = (U * eps_bar[:, j]) @ U.conj().T
        for R in h:
            out[R] += _phase(k, R, -1) * Hk
    return out


def hermitian_direction(h, rng):
    """Random perturbation with dH_{-R} = dH_R^H (and dH_0 Hermitian)."""
    n = next(iter(h.values())).shape[0]
    d = {}
    for R in h:
        if R in d:
            continue
        mR = tuple(-x for x in R)
        X = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        if mR == R:
            d[R] = 0.5 * (X + X.conj().T)
        else:
            d[R] = X
            if mR in h:
                d[mR] = X.conj().T
    return d


def pairing(A, B):
    """Re sum_R <A_R, B_R>."""
    return float(sum(np.real(np.vdot(A[R], B[R])) for R in A if R in B))


# ---------------------------------------------------------------- converged Hartree-Fock SCF
def grand_potential(bands, w, mu, T):
    """Omega_band = -T sum_k w_k sum_j log(1 + e^{-(eps_j - mu)/T}) (T = 0: sum of eps - mu
    below mu) and N = sum_k w_k sum_j f_j, for bands (n, nk)."""
    x = bands - mu
    if T > 0:
        y = x / T
        om = -T * np.where(y > 0, np.log1p(np.exp(-np.abs(y))), -y + np.log1p(np.exp(-np.abs(y))))
    else:
        om = np.minimum(x, 0.0)
    f = K.fermidirac(bands, mu, T)
    return float(np.sum(w[None, :] * om)), float(np.sum(w[None, :] * f))


def free_energy(hf, ks, w, mu, T):
    """F = Omega_band(hMF) + mu N - (eH + eF + eJ) of a HartreeFock evaluated at rho
    (Meanfield/hartreefock.jl:236 double counting; the Mermin free energy of the
    mean-field bands at the filling's chemical potential)."""
    bands, _ = K.bandmatrix(hf.hMF, ks)
    om, ne = grand_potential(bands, w, mu, T)
    return om + mu * ne - hf.doublecounting(), om, ne


def hf_transpose(hf, gbar, rho_keys):
    """Phi^T of the linear part of hMF(rho): Fock -v .* rho at the keys of v present in rho
    (cotangent -conj(v_L) .* gbar_L), Hartree diag(V0 diag rho_0) (cotangent on the
    diagonal of rho_0: Re sum_i conj(V0[i, j]) gbar_0[i, i]); Meanfield/hartreefock.jl:247-289."""
    n = hf.V0.shape[0]
    out = {L: np.zeros((n, n), complex) for L in rho_keys}
    if hf.fock:
        for L in rho_keys:
            if L in hf.v and L in gbar:
                out[L] = -np.conj(hf.v[L]) * gbar[L]
    z = tuple(0 for _ in next(iter(rho_keys)))
    if hf.hartree:
        s = np.real(np.conj(hf.V0).T @ np.diag(gbar[z]))
        out[z] = out[z] + np.diag(s)
    return out


def scf_band_loss_gradient(h, v, ks, w, mu, T, rho, eps_bar, beta=0.3, tol=1e-12, maxiter=2000):
    """dL/dh_R through the converged SCF for a loss of the mean-field bands (cotangent
    eps_bar, (n, nk)): gbar = bands VJP at hMF, z = D'^T Phi^T (gbar + z) with
    D'^T(G) = VJP_mu(G) - (Re tr VJP_mu(G)_0 / Re tr Nbar_0) Nbar, Nbar the cotangent of
    the electron count, solved by damped iteration; returns (gbar + z on the keys of h,
    residual, iterations)."""
    from .meanfield import HartreeFock
    hf = HartreeFock(h, v)
    hf(rho)
    hmf = hf.hMF
    z0 = tuple(0 for _ in next(iter(h)))
    gbar = bands_vjp(hmf, ks, eps_bar)
    if T > 0:
        bands, _ = K.bandmatrix(hmf, ks)
        x = bands - mu
        fm = K.fermidirac(bands, mu, T)
        slope = -fm * (1.0 - fm) / T
        Nbar = bands_vjp(hmf, ks, w[None, :] * slope)
        c = float(np.real(np.trace(Nbar[z0])))
    else:
        Nbar, c = None, 0.0
    z = {R: np.zeros_like(M) for R, M in gbar.items()}
    res, it = np.inf, 0
    for it in range(1, maxiter + 1):
        gin = {R: gbar[R] + z[R] for R in gbar}
        rbar = hf_transpose(hf, gin, list(rho.keys()))
        Hb = densitymatrix_vjp(hmf, ks, w, mu, T, rbar)
        t = float(np.real(np.trace(Hb[z0])))
        r = t / c if c != 0.0 else 0.0
        dn = nz = 0.0
        for R in z:
            zn = Hb[R] - (r * Nbar[R] if Nbar is not None else 0.0)
            y = (1 - beta) * z[R] + beta * zn
            dn += np.sum(np.abs(y - z[R]) ** 2)
            nz += np.sum(np.abs(y) ** 2)
            z[R] = y
        res = math.sqrt(dn) / math.sqrt(nz) if nz > 0 else math.sqrt(dn)
        if res < tol:
            break
    return {R: gbar[R] + z[R] for R in h}, res, it
