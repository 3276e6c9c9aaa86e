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
