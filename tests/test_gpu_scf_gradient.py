"""Derivatives of the converged Hartree-Fock SCF through the C ABI (lqm_scf_hf_gradient).

* n = 8 (triangular Hubbard, 2 x 2 spinful, 4 x 4 k): the free energy, dF/dh and the
  implicit-function gradient of a band-fit loss against the oracle's restatement
  (oracle/adjoint.py, itself pinned to finite differences in
  test_scf_gradient_oracle.py), at the device SCF's converged rho and mu, to 1e-9.
* n = 72 (the 6 x 6 spinful triangular Hubbard model, 36 x 36 k-points, T = 0.02,
  U = 4): the gradients of F and of the band-fit loss with respect to the hopping
  scalings t, t' and a per-site field, against FP64 central finite differences
  (step 1e-6) of the device SCF converged to 1e-13, to 1e-6 relative.
"""
import numpy as np
import pytest

from lqm_workloads import lattice as L
from lqm_workloads import models as M
from oracle import adjoint as A
from oracle import kspace as K
from oracle import meanfield as MF
from test_scf_gradient_oracle import band_target, hubbard_family

pytestmark = pytest.mark.gpu


def _scf(lqm, ctx, h, v, r0, ks, T, tol):
    res = lqm.solvehartreefock(h, v, r0, 0.5, ks, T=T, beta=0.3, tol=tol, iterations=3000, acceleration="anderson",
                               anderson_depth=5, ctx=ctx)
    assert res.converged, res.residual
    return res


def test_scf_gradient_matches_oracle_n8(lqm, ctx):
    lat, v, h_of, dirs = hubbard_family(L_super=2)
    ks = L.regulargrid(4 * 4)
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    T = 0.05
    h = h_of(np.array([-1.0, 0.2, 0.1]))
    res = _scf(lqm, ctx, h, v, {(0, 0): M.random_local_magnetization(lat.norb, seed=5)}, ks, T, 1e-14)
    rho, mu = res.rho, res.mf.mu
    hf = MF.HartreeFock(h, v)
    hf(rho)
    bands0, _ = K.bandmatrix(hf.hMF, ks)
    eps_bar = w[None, :] * (bands0 - band_target(bands0))
    g = lqm.scf_hf_gradient(h, v, rho, mu, ks, T=T, eps_bar=eps_bar, beta=0.3, tol=1e-13, ctx=ctx)
    F_ref = A.free_energy(hf, ks, w, mu, T)[0]
    dF_ref, _ = K.densitymatrix(hf.hMF, ks, w, mu, T, list(h.keys()))
    dL_ref, _, _ = A.scf_band_loss_gradient(h, v, ks, w, mu, T, rho, eps_bar, beta=0.3, tol=1e-13)
    assert g.residual < 1e-13
    assert abs(g.F - F_ref) <= 1e-10 * max(1.0, abs(F_ref))
    assert max(np.max(np.abs(g.dF_dh[R] - dF_ref[R])) for R in h) <= 1e-9
    scale = max(np.max(np.abs(dL_ref[R])) for R in h)
    assert max(np.max(np.abs(g.dL_dh[R] - dL_ref[R])) for R in h) <= 1e-9 * max(1.0, scale)


def test_scf_gradient_c4_matches_finite_differences(lqm, ctx):
    lat, v, h_of, dirs = hubbard_family(L_super=6)
    assert v[(0, 0)].shape[0] == 72
    ks = L.regulargrid(36 * 36)
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    T = 0.02
    th0 = np.array([-1.0, 0.2, 0.1])
    h = h_of(th0)
    base = _scf(lqm, ctx, h, v, {(0, 0): M.random_local_magnetization(lat.norb, seed=7)}, ks, T, 1e-13)
    rho, mu = base.rho, base.mf.mu
    hmf, _, _, _ = lqm.hartreefock_eval(h, v, rho, ctx=ctx)
    bands0, _ = lqm.bandmatrix(hmf, ks, ctx=ctx)
    target = band_target(bands0)
    g = lqm.scf_hf_gradient(h, v, rho, mu, ks, T=T, eps_bar=w[None, :] * (bands0 - target), beta=0.3, tol=1e-12,
                            ctx=ctx)
    assert g.residual < 1e-12

    def values(th):
        hh = h_of(th)
        r = _scf(lqm, ctx, hh, v, rho, ks, T, 1e-13)
        F = lqm.scf_hf_gradient(hh, v, r.rho, r.mf.mu, ks, T=T, ctx=ctx).F
        hm, _, _, _ = lqm.hartreefock_eval(hh, v, r.rho, ctx=ctx)
        b, _ = lqm.bandmatrix(hm, ks, ctx=ctx)
        return F, 0.5 * float(np.sum(w[None, :] * (b - target) ** 2))

    d = 1e-6
    for p, dh in enumerate(dirs):
        e = np.zeros(3)
        e[p] = d
        Fp, Lp = values(th0 + e)
        Fm, Lm = values(th0 - e)
        fdF, fdL = (Fp - Fm) / (2 * d), (Lp - Lm) / (2 * d)
        gF, gL = A.pairing(g.dF_dh, dh), A.pairing(g.dL_dh, dh)
        assert abs(gF - fdF) <= 1e-6 * max(abs(fdF), 1e-3), (p, gF, fdF)
        assert abs(gL - fdL) <= 1e-6 * max(abs(fdL), 1e-3), (p, gL, fdL)
