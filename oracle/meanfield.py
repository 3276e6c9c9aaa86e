"""Hartree-Fock SCF restated from LatticeQM.jl (oracle; test infrastructure only)."""
import math

import numpy as np

from . import kspace as K


class ExchangeKernel:
    """Meanfield/hartreefock.jl:24-76 (ExchangeKernel) with 0-based sites and flavors:
    j a site-space Hops, sf2idx[a, f] the orbital of (site a, flavor f), Jtot = sum_L j[L]."""

    def __init__(self, j, siteof, flavorof):
        siteof, flavorof = list(siteof), list(flavorof)
        if len(siteof) != len(flavorof):
            raise ValueError("siteof and flavorof must have equal length")
        ns, nf = max(siteof) + 1, max(flavorof) + 1
        z = tuple(0 for _ in next(iter(j.keys())))
        if j[z].shape[0] != ns:
            raise ValueError("exchange kernel dimension does not match the number of sites")
        if np.any(np.diag(j[z]) != 0):
            raise ValueError("onsite self-exchange j[0][a,a] must be zero")
        sf = -np.ones((ns, nf), int)
        for I, (a_, f_) in enumerate(zip(siteof, flavorof)):
            if sf[a_, f_] >= 0:
                raise ValueError("duplicate (site, flavor)")
            sf[a_, f_] = I
        if np.any(sf < 0):
            raise ValueError("every (site, flavor) pair must appear once")
        self.j = {L: np.asarray(M, complex) for L, M in j.items()}
        self.sf2idx = sf
        self.Jtot = sum(self.j[L] for L in self.j)


class HartreeFock:
    """Meanfield/hartreefock.jl:143-175 (struct), :184-228 (call), :247-289 (fields),
    :298-381 (exchange), :392-410 (energies)."""

    def __init__(self, h, v, hartree=True, fock=True, exchange=None):
        self.h = h
        self.v = v
        self.hartree, self.fock, self.exchange = hartree, fock, exchange
        self.V0 = sum(v[L] for L in v)  # hartreefock.jl:159
        keys = list(h.keys()) + [L for L in v if L not in h]
        n = next(iter(h.values())).shape[0]
        self.hMF = {L: np.zeros((n, n), complex) for L in keys}
        self.mu = 0.0
        self.eH = self.eF = self.eJ = self.eband = self.ekin = 0.0

    def __call__(self, rho):
        n = next(iter(self.h.values())).shape[0]
        # initialize_hMF! (hartreefock.jl:191-205)
        for L in self.hMF:
            self.hMF[L] = np.zeros((n, n), complex)
        for L in self.h:
            self.hMF[L] = self.hMF[L] + self.h[L]
        z = tuple(0 for _ in next(iter(rho.keys())))
        # Fock: hMF[L] -= v[L] .* rho[L] (hartreefock.jl:247-276)
        if self.fock:
            for L in self.v:
                if L in rho:
                    self.hMF[L] = self.hMF[L] - self.v[L] * rho[L]
        # Hartree: hMF[0][i,i] += (V0 diag rho0)_i (hartreefock.jl:278-289)
        if self.hartree:
            d = self.V0 @ np.diag(rho[z])
            self.hMF[z] = self.hMF[z] + np.diag(d)
        if self.exchange is not None:
            self._add_exchange(rho, z)
        # energies (hartreefock.jl:345-410)
        nv = np.diag(rho[z])
        self.eH = float(np.real(0.5 * (nv @ self.V0 @ nv))) if self.hartree else 0.0
        self.eF = float(np.real(-0.5 * sum(np.sum(rho[L] * np.conj(rho[L]) * vL)
                                           for L, vL in self.v.items() if L in rho))) if self.fock else 0.0
        self.eJ = self._exchange_energy(rho, z) if self.exchange is not None else 0.0
        return self

    def _add_exchange(self, rho, z):
        """meanfieldOperator_addexchange! (hartreefock.jl:298-337)."""
        ek = self.exchange
        ix = ek.sf2idx
        ns, nf = ix.shape
        H0, r0 = self.hMF[z], rho[z]
        for a in range(ns):
            for b in range(ns):
                J = ek.Jtot[a, b]
                if J == 0:
                    continue
                for al in range(nf):
                    for be in range(nf):
                        H0[ix[a, al], ix[a, be]] -= J * r0[ix[b, al], ix[b, be]]
        n = H0.shape[0]
        for L, jL in ek.j.items():
            if L not in rho:
                continue
            if L not in self.hMF:
                self.hMF[L] = np.zeros((n, n), complex)
            hL, rL = self.hMF[L], rho[L]
            for a in range(ns):
                for b in range(ns):
                    J = jL[a, b]
                    if J == 0:
                        continue
                    tau = sum(rL[ix[a, al], ix[b, al]] for al in range(nf))
                    for al in range(nf):
                        hL[ix[a, al], ix[b, al]] += J * tau

    def _exchange_energy(self, rho, z):
        """exchange_energy (hartreefock.jl:345-381)."""
        ek = self.exchange
        ix = ek.sf2idx
        ns, nf = ix.shape
        r0 = rho[z]
        e = 0.0 + 0.0j
        for a in range(ns):
            for b in range(ns):
                J = ek.Jtot[a, b]
                if J == 0:
                    continue
                s = sum(r0[ix[a, al], ix[a, be]] * r0[ix[b, be], ix[b, al]] for al in range(nf) for be in range(nf))
                e -= J * s / 2
        for L, jL in ek.j.items():
            if L not in rho:
                continue
            rL = rho[L]
            for a in range(ns):
                for b in range(ns):
                    J = jL[a, b]
                    if J == 0:
                        continue
                    tau = sum(rL[ix[a, al], ix[b, al]] for al in range(nf))
                    e += J * abs(tau) ** 2 / 2
        return float(np.real(e))

    def doublecounting(self):
        return self.eH + self.eF + self.eJ  # hartreefock.jl:236


def hermitianize(rho):
    # TightBinding/types.jl:174-189
    for R in list(rho.keys()):
        mR = tuple(-x for x in R)
        if mR in rho:
            rho[R] = (rho[R] + rho[mR].conj().T) / 2
            rho[mR] = rho[R].conj().T.copy()
        else:
            rho[mR] = rho[R].conj().T.copy()
    return rho


def is_hermitian(rho, tol=np.sqrt(np.finfo(float).eps)):
    # TightBinding/types.jl:165-172
    for R in rho:
        mR = tuple(-x for x in R)
        if mR not in rho or np.max(np.abs(rho[R] - rho[mR].conj().T)) >= tol:
            return False
    return True


def anderson_update(flat_x, flat_f, hist_x, hist_f, beta):
    """fixedpoint.jl:201-231 (_anderson_update): Type-II update with damping beta;
    plain damped mixing without history or for a non-finite least-squares solution.
    The least-squares solve `dG \\ g` is restated with numpy's lstsq (the same
    solution for a full-rank history)."""
    m = len(hist_x) - 1
    if m == 0:
        return beta * flat_f + (1 - beta) * flat_x
    dX = np.stack([hist_x[i + 1] - hist_x[i] for i in range(m)], axis=1)
    dF = np.stack([hist_f[i + 1] - hist_f[i] for i in range(m)], axis=1)
    dG = dF - dX
    g = flat_f - flat_x
    gamma = np.linalg.lstsq(dG, g, rcond=None)[0]
    if not np.all(np.isfinite(gamma)):
        return beta * flat_f + (1 - beta) * flat_x
    return (1 - beta) * flat_x + beta * flat_f - ((1 - beta) * dX + beta * dF) @ gamma


def _flatten(rho, keys):
    return np.concatenate([rho[k].ravel(order="F") for k in keys])


def _unflatten(rho, flat, keys):
    off = 0
    for k in keys:
        sz = rho[k].size
        rho[k] = flat[off:off + sz].reshape(rho[k].shape, order="F").copy()
        off += sz


def commutator_kspace_norm(H, rho, ks, w=None):
    """Meanfield/selfconsistent.jl:130-166: sqrt(sum_k w_k ||H(k) rho(k) - rho(k) H(k)||_F^2),
    w = 1/nk by default."""
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk) if w is None else w
    s = 0.0
    for j in range(nk):
        Hk = K.fouriersum(H, ks[:, j])
        Rk = K.fouriersum(rho, ks[:, j])
        C = Hk @ Rk - Rk @ Hk
        s += w[j] * float(np.sum(np.abs(C) ** 2))
    return math.sqrt(s)


def enrichkeys(rho, klin):
    """Meanfield/initialguess.jl:262-277 (enrichkeys!): add zero blocks for every key of
    {-klin//2 .. klin//2}^d (first index fastest) that rho lacks."""
    sample = next(iter(rho.values()))
    d = len(next(iter(rho.keys())))
    Lmax = klin // 2
    for L in _product_first_fastest([range(-Lmax, Lmax + 1)] * d):
        if L not in rho:
            rho[L] = np.zeros_like(sample)
    return rho


def _product_first_fastest(ranges):
    out = [()]
    for r in ranges:
        out = [o + (x,) for x in r for o in out]
    return out


def solvehartreefock(h, v, rho_init, filling, ks, T=0.0, beta=1.0, tol=1e-7,
                     iterations=500, log=None, acceleration="linear", anderson_depth=5,
                     residual_norm="density", hartree=True, fock=True, exchange=None):
    """solvehartreefock -> _scf_driver! -> fixedpoint!.

    Meanfield/selfconsistent.jl:19,62-69,256-336,366-381 and fixedpoint.jl:39-194.
    Each iteration: hf(rho0); mu from the eigenvalues of hMF on every k;
    rho1 = getdensitymatrix!(hMF, mu); linear mixing (or, with
    acceleration="anderson", the Anderson update of fixedpoint.jl:64-142 with
    its Hermitian projection) and the relative residual (or, with
    residual_norm="commutator", ||[hMF, rho0]|| of selfconsistent.jl:399-405)."""
    use_anderson = acceleration == "anderson" and anderson_depth > 0
    hist_x, hist_f = [], []
    rho0 = {L: M.copy() for L, M in rho_init.items()}
    if not is_hermitian(rho0):
        hermitianize(rho0)
    rho1 = {L: M.copy() for L, M in rho0.items()}
    hf = HartreeFock(h, v, hartree=hartree, fock=fock, exchange=exchange)
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk)
    converged = False
    residual = np.inf
    E = 0.0
    it = 0
    while it < iterations:
        it += 1
        hf(rho0)
        comm = commutator_kspace_norm(hf.hMF, rho0, ks) if residual_norm == "commutator" else None
        bands, _ = K.bandmatrix(hf.hMF, ks)
        hf.mu = K.chemicalpotential(bands, filling, T)
        rho_new, eband = K.densitymatrix(hf.hMF, ks, w, hf.mu, T, list(rho1.keys()))
        rho1 = rho_new
        hf.eband = eband
        hf.ekin = eband - 2 * hf.doublecounting()
        E = eband - hf.doublecounting()
        if use_anderson:  # fixedpoint.jl:101-142
            keys = sorted(rho0.keys())
            fx, ff = _flatten(rho0, keys), _flatten(rho1, keys)
            hist_x.append(fx.copy())
            hist_f.append(ff.copy())
            while len(hist_x) > anderson_depth + 1:
                hist_x.pop(0)
                hist_f.pop(0)
            _unflatten(rho1, anderson_update(fx, ff, hist_x, hist_f, beta), keys)
            hermitianize(rho1)
            fn = _flatten(rho1, keys)
            diff = np.linalg.norm(fn - fx)
            nrm = np.linalg.norm(fn)
        else:
            for L in rho0:  # fixedpoint.jl:146-148
                rho1[L] = beta * rho1[L] + (1 - beta) * rho0[L]
            diff = np.linalg.norm([np.linalg.norm(rho1[L] - rho0[L]) for L in rho0])
            nrm = np.linalg.norm([np.linalg.norm(rho1[L]) for L in rho0])
        residual = diff / nrm if nrm > np.finfo(float).eps else diff
        if comm is not None:  # selfconsistent.jl:399-405, evaluated before the mixing
            residual = comm
        for L in rho0:
            rho0[L] = rho1[L].copy()
        if log is not None:
            log(it, E, residual, hf.ekin, hf.eband, hf.eH, hf.eF, hf.mu)
        if residual < tol:
            converged = True
            break
    hf(rho1)  # selfconsistent.jl:326-328
    hf.ekin = hf.eband - 2 * hf.doublecounting()
    E = hf.eband - hf.doublecounting()
    if not is_hermitian(rho1):
        hermitianize(rho1)
    return rho1, E, hf, converged, residual, it
