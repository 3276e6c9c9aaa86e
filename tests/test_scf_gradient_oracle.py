"""The oracle's derivatives of the converged Hartree-Fock SCF against central finite
differences (CPU; pins oracle/adjoint.py before the device gradient is compared with it).

Model: the spinful triangular Hubbard model on a 2 x 2 supercell (n = 8), 4 x 4 k-points,
T = 0.05, filling 0.5; h(theta) = t P_NN + t' P_NNN + m sigma_z(site 0), theta = (t, t', m)
(the hopping-shell scalings and a per-site field).  The SCF (Meanfield/selfconsistent.jl:
256-336, restated in oracle/meanfield.py) is converged to a relative residual of 1e-14:
* the free energy F = Omega_band + mu N - (eH + eF): dF/dtheta = Re <rho*, dh/dtheta>;
* a band-fit loss L = 1/2 sum_k w_k sum_j (eps_jk(hMF*) - target_jk)^2: the implicit-
  function adjoint through the fixed point, including the chemical potential's response.
FD step 1e-6, agreement to 1e-6 relative.
"""
import math

import numpy as np

from lqm_workloads import lattice as L
from lqm_workloads import models as M
from oracle import adjoint as A
from oracle import kspace as K
from oracle import meanfield as MF


def hubbard_family(L_super=2):
    """h(theta) for theta = (t, t', m) and its derivative directions."""
    lat, _, v = M.triangular_hubbard(L_super=L_super)
    P1 = M.addspin(M.nearestneighbor(lat, 1.0, a=1.0))
    P2 = M.addspin(M.nearestneighbor(lat, 1.0, a=math.sqrt(3.0)))
    n = 2 * lat.norb
    z = (0, 0)
    Z0 = {z: np.diag([1.0, -1.0] + [0.0] * (n - 2)).astype(complex)}
    keys = list(P1.keys()) + [R for R in P2 if R not in P1]
    if z not in keys:
        keys.append(z)

    def h_of(th):
        t, tp, m = th
        return {R: t * P1.get(R, 0) + tp * P2.get(R, 0) + m * Z0.get(R, 0) + np.zeros((n, n), complex) for R in keys}

    dirs = [{R: P1.get(R, np.zeros((n, n))) + 0j for R in keys}, {R: P2.get(R, np.zeros((n, n))) + 0j for R in keys},
            {R: Z0.get(R, np.zeros((n, n))) + 0j for R in keys}]
    return lat, v, h_of, dirs


def band_target(bands0):
    # a smooth function of the bands, so that degenerate levels share their target
    return bands0 - 0.05 - 0.02 * bands0


def test_oracle_scf_gradients_match_finite_differences():
    lat, v, h_of, dirs = hubbard_family()
    ks = L.regulargrid(4 * 4)
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    T, fill, beta = 0.05, 0.5, 0.3
    th0 = np.array([-1.0, 0.2, 0.1])

    def scf(th, r0):
        rho, E, hf, conv, res, it = MF.solvehartreefock(h_of(th), v, r0, fill, ks, T=T, beta=beta, tol=1e-14,
                                                        iterations=5000, acceleration="anderson", anderson_depth=5)
        assert conv
        return rho, hf

    rho, hf = scf(th0, {(0, 0): M.random_local_magnetization(lat.norb, seed=5)})
    mu = hf.mu
    h0 = h_of(th0)
    dF_dh, _ = K.densitymatrix(hf.hMF, ks, w, mu, T, list(h0.keys()))
    bands0, _ = K.bandmatrix(hf.hMF, ks)
    target = band_target(bands0)
    gL, res, _ = A.scf_band_loss_gradient(h0, v, ks, w, mu, T, rho, w[None, :] * (bands0 - target), beta=beta,
                                          tol=1e-13)
    assert res < 1e-13

    def loss(hf_):
        b, _ = K.bandmatrix(hf_.hMF, ks)
        return 0.5 * float(np.sum(w[None, :] * (b - target) ** 2))

    d = 1e-6
    for p, dh in enumerate(dirs):
        e = np.zeros(3)
        e[p] = d
        _, hp = scf(th0 + e, rho)
        _, hm = scf(th0 - e, rho)
        fdF = (A.free_energy(hp, ks, w, hp.mu, T)[0] - A.free_energy(hm, ks, w, hm.mu, T)[0]) / (2 * d)
        fdL = (loss(hp) - loss(hm)) / (2 * d)
        gF = A.pairing(dF_dh, dh)
        gl = A.pairing(gL, dh)
        assert abs(gF - fdF) <= 1e-6 * max(abs(fdF), 1e-3), (p, gF, fdF)
        assert abs(gl - fdL) <= 1e-6 * max(abs(fdL), 1e-3), (p, gl, fdL)
