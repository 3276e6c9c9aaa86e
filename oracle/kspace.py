"""k-space hot path restated from LatticeQM.jl (oracle; test infrastructure only)."""
import math
import struct

import numpy as np
import scipy.linalg as sla


def fouriersum(h, k):
    """H(k) = sum_R H_R exp(+i 2 pi k.R), summed in dict order.

    TightBinding/types.jl:8 (fourierphase) and :18-25 (fouriersum!)."""
    k = np.atleast_1d(np.asarray(k, float))
    out = None
    for R, M in h.items():
        ph = np.exp(1j * 2 * math.pi * float(np.dot(k, np.array(R, float))))
        out = M * ph if out is None else out + M * ph
    return out


def eigh_upper(Hk, vectors=True):
    """LAPACK zheevr on the upper triangle, all pairs, ascending.

    Eigen/Eigen.jl:22-23,32 (``eigen!(Hermitian(M))``, upper triangle), which
    LinearAlgebra maps to ``zheevr`` (extra/benchmarks/bench_heevr.jl:38,68)."""
    if vectors:
        return sla.eigh(Hk, lower=False, driver="evr")
    return sla.eigh(Hk, lower=False, driver="evr", eigvals_only=True)


def bandmatrix(h, ks, vectors=False):
    """bands (n, nk), optionally U (nk, n, n); Spectrum/bands.jl:164-227."""
    n = next(iter(h.values())).shape[0]
    nk = ks.shape[1]
    bands = np.zeros((n, nk))
    U = np.zeros((nk, n, n), complex) if vectors else None
    for j in range(nk):
        Hk = fouriersum(h, ks[:, j])
        if vectors:
            e, u = eigh_upper(Hk, True)
            U[j] = u
        else:
            e = eigh_upper(Hk, False)
        bands[:, j] = e
    return bands, U


def bandmatrix_obs(h, ks, projectors):
    """bands (n, nk) and obs (n, nk, nproj): obs[i, j, p] = Re <u_i| O_p(k_j) |u_i>;
    Spectrum/bands.jl:52-60 (ExpvalMap: a matrix, or a k-dependent operator, here a
    Hops dict Bloch-summed like H), :107-112 (compute_bandexpvals!), :212-227."""
    n = next(iter(h.values())).shape[0]
    nk = ks.shape[1]
    bands = np.zeros((n, nk))
    obs = np.zeros((n, nk, len(projectors)))
    for j in range(nk):
        k = ks[:, j]
        e, U = eigh_upper(fouriersum(h, k), True)
        bands[:, j] = e
        for p, op in enumerate(projectors):
            O = fouriersum(op, k) if isinstance(op, dict) else np.asarray(op)
            obs[:, j, p] = np.real(np.einsum("ri,rs,si->i", U.conj(), O, U))
    return bands, obs


def density(h, ks, mu=0.0):
    """Spectrum/dos.jl:20-52: n_i = 1/L sum_k sum_{eps_j <= mu} |U_ij|^2."""
    n = next(iter(h.values())).shape[0]
    out = np.zeros(n)
    for j in range(ks.shape[1]):
        e, U = eigh_upper(fouriersum(h, ks[:, j]), True)
        out += np.sum(np.abs(U[:, e <= mu]) ** 2, axis=1)
    return out / ks.shape[1]


def ldos(h, ks, omegas, gamma=0.1):
    """Spectrum/dos.jl:56-98: n_i = 1/(L pi) sum_k sum_j |U_ij|^2 (1/F) sum_w
    Gamma / ((w - eps_j)^2 + Gamma^2) (the k-point's frequency average counted once)."""
    omegas = np.atleast_1d(np.asarray(omegas, float))
    n = next(iter(h.values())).shape[0]
    out = np.zeros(n)
    for j in range(ks.shape[1]):
        e, U = eigh_upper(fouriersum(h, ks[:, j]), True)
        a = np.mean(gamma / ((omegas[:, None] - e[None, :]) ** 2 + gamma ** 2), axis=0)
        out += (np.abs(U) ** 2) @ a
    return out / (ks.shape[1] * np.pi)


def fermisurfacedensity_fromdata(bands, energies, obs=None, broadening="auto"):
    """Spectrum/fermisurface.jl (fermisurfacedensity_fromdata, getbroadening): per energy
    and k, sum_b (1/pi) w g^2 / (g^2 + (eps - E)^2); :auto g = mean_b std_k(eps_b) / sqrt(nk)
    (std with n - 1)."""
    bands = np.asarray(bands, float)
    energies = np.atleast_1d(np.asarray(energies, float))
    if not isinstance(broadening, (int, float)) or broadening == "auto":
        broadening = float(np.mean([np.std(b, ddof=1) for b in bands])) / math.sqrt(bands.shape[1])
    g2 = broadening ** 2
    out = np.zeros((len(energies), bands.shape[1]))
    for j in range(bands.shape[1]):
        t = (1 / math.pi) * g2 / (g2 + (bands[:, j][:, None] - energies[None, :]) ** 2)
        if obs is not None:
            t = obs[:, j][:, None] * t
        out[:, j] = np.sum(t, axis=0)
    return out, broadening


def berry(h, NX, NY, bands):
    """Spectrum/berry.jl:48-82 (statesgrid on range(0,1,N) x range(0,1,N) + 1.34e-8)
    and :107-137 (link L = det(A^H B)/|det|, plaquette phase real(log(...)/(2 pi i)));
    0-based band indices; F (NX-1, NY-1)."""
    S = {}
    for j in range(NY):
        for i in range(NX):
            k = np.array([i / (NX - 1), j / (NY - 1)]) + 1.34e-8
            _, U = eigh_upper(fouriersum(h, k), True)
            S[i, j] = U[:, list(bands)]

    def link(A, B):
        d = np.linalg.det(A.conj().T @ B)
        return d / abs(d)

    F = np.zeros((NX - 1, NY - 1))
    for i in range(NX - 1):
        for j in range(NY - 1):
            z = link(S[i, j], S[i + 1, j]) * link(S[i + 1, j], S[i + 1, j + 1]) \
                / link(S[i, j + 1], S[i + 1, j + 1]) / link(S[i, j], S[i, j + 1])
            F[i, j] = np.real(np.log(z) / (2j * math.pi))
    return F


def kubo(omegas, e, U, A, B, mu=0.0, gamma=0.025, T=0.1):
    """LinearResponse/kubo.jl:11-26 (kubo!): sum_{i != j} (f_i - f_j) M_ij /
    ((e_i - e_j) - (w + i Gamma)) with M = (U^H A U) .* transpose(U^H B U), the pairs
    in the reference's order (i fastest)."""
    omegas = np.asarray(omegas, float)
    M = (U.conj().T @ A @ U) * (U.conj().T @ B @ U).T
    fd = fermidirac(e, mu, T)
    out = np.zeros(len(omegas), complex)
    n = len(e)
    for j in range(n):
        for i in range(n):
            if i != j:
                out += (fd[i] - fd[j]) * M[i, j] / ((e[i] - e[j]) - (omegas + 1j * gamma))
    return out


def opticalconductivity(omegas, h, J1, J2, ks, mu=0.0, gamma=0.025, T=0.1):
    """LinearResponse/opticalconductivity.jl:101-127: chi(w) = -(i/N) sum_k
    kubo!(w, e_k, U_k, J1(k), J2(k)^H)."""
    out = np.zeros(len(np.atleast_1d(omegas)), complex)
    for j in range(ks.shape[1]):
        k = ks[:, j]
        e, U = eigh_upper(fouriersum(h, k), True)
        out += kubo(np.atleast_1d(omegas), e, U, fouriersum(J1, k), fouriersum(J2, k).conj().T, mu, gamma, T)
    return out * (-1j / ks.shape[1])


def _rot2(t):
    # Structure/rotate.jl:8
    return np.array([[math.cos(t), -math.sin(t)], [math.sin(t), math.cos(t)]])


def berryalongpath(h, kpoints):
    """Spectrum/berry.jl:170-238: per band and path point the abelian plaquette phase of
    the corners kc + dR, dU, dD, dL (padded path, shifted by 1.34e-6 |k2 - k1| (1, 1/sqrt2))."""
    kpoints = np.asarray(kpoints, float)
    N = kpoints.shape[1]
    n = next(iter(h.values())).shape[0]
    k0 = kpoints[:, 0] - (kpoints[:, 1] - kpoints[:, 0])
    kN1 = kpoints[:, N - 1] + (kpoints[:, N - 1] - kpoints[:, N - 2])
    kp = np.hstack([k0[:, None], kpoints, kN1[:, None]])
    kp = kp + 1.34e-6 * np.linalg.norm(kp[:, 1] - kp[:, 0]) * np.array([1.0, 0.7071067811865476])[:, None]
    out = np.zeros((n, N))

    def link(a, b):
        z = np.vdot(a, b)
        return z / abs(z)

    for j in range(N):
        kc = kp[:, j + 1]
        dR = (kp[:, j + 2] - kc) / 2
        dL = (kp[:, j] - kc) / 2
        dU = (_rot2(math.pi / 2) @ dR + _rot2(-math.pi / 2) @ dL) / 2
        dD = (_rot2(-math.pi / 2) @ dR + _rot2(math.pi / 2) @ dL) / 2
        Us = [eigh_upper(fouriersum(h, kc + dk), True)[1] for dk in (dR, dU, dD, dL)]
        for i in range(n):
            R, U, D, Lf = (X[:, i] for X in Us)
            z = link(R, U) * link(U, Lf) / link(D, Lf) / link(R, D)
            out[i, j] = np.real(np.log(z) / (2j * math.pi))
    return out


def berry_grid(NX, NY):
    """k-points of statesgrid (Spectrum/berry.jl:49-82): range(0, 1, length=N) per
    direction, first index fastest, + 1.34e-8."""
    return np.array([[i / (NX - 1), j / (NY - 1)] for j in range(NY) for i in range(NX)]).T + 1.34e-8


def getcherns(h, NX, NY=0, bands=None):
    """getcherns(H, NX, NY, bands) (Spectrum/berry.jl:378-382): per band the summed
    plaquette phases of its single-band state grid (bands 0-based; all when None)."""
    NY = NX if NY < 1 else NY
    n = next(iter(h.values())).shape[0]
    bands = list(range(n)) if bands is None else list(bands)
    return [float(np.sum(berry(h, NX, NY, [b]))) for b in bands]


def spectralgaps(h, NX, NY=0, gaptol=1e-6):
    """spectralgaps(H, NX, NY; gaptol) (Spectrum/berry.jl:421-442): gaps between the
    grid maximum of band n and the grid minimum of band n+1 wider than gaptol, as
    (n, elo, ehi) with n the number of bands below (1-based count)."""
    NY = NX if NY < 1 else NY
    E, _ = bandmatrix(h, berry_grid(NX, NY))
    emin, emax = E.min(axis=1), E.max(axis=1)
    return [(m + 1, float(emax[m]), float(emin[m + 1])) for m in range(E.shape[0] - 1)
            if emin[m + 1] - emax[m] > gaptol]


def gapcherns(h, NX, NY=0, gaptol=1e-6):
    """gapcherns(H, NX, NY; gaptol) (Spectrum/berry.jl:470-487): (n, elo, ehi, chern) per
    gap, chern = round(sum(berry(states[:, :, :, 1:n])))."""
    NY = NX if NY < 1 else NY
    return [(m, lo, hi, int(round(float(np.sum(berry(h, NX, NY, list(range(m)))))))) for m, lo, hi in
            spectralgaps(h, NX, NY, gaptol)]


def statesgrid(h, NX, NY, bands):
    """statesgrid(H, NX, NY, bandindices) (Spectrum/berry.jl:49-82): S[i, j] = the n x nb
    eigenvector columns at k = (i/(NX-1), j/(NY-1)) + 1.34e-8."""
    n = next(iter(h.values())).shape[0]
    S = np.zeros((NX, NY, n, len(bands)), complex)
    for i in range(NX):
        for j in range(NY):
            k = np.array([i / (NX - 1), j / (NY - 1)]) + 1.34e-8
            _, U = eigh_upper(fouriersum(h, k), True)
            S[i, j] = U[:, list(bands)]
    return S


def wilson1d(grid3):
    """Wilson1D(statesgrid (NY, M1, M2)) (Spectrum/berry.jl:312-327, j0 = 0): F = prod over the
    periodic links of U V^H from svd(S_j^H S_{j+1}); eigenphases angle/(2 pi) ascending."""
    NY = grid3.shape[0]
    m = grid3.shape[2]
    F = np.eye(m, dtype=complex)
    for j in range(NY):
        A = grid3[j].conj().T @ grid3[(j + 1) % NY]
        Us, _, Vh = np.linalg.svd(A)
        F = F @ (Us @ Vh)
    ev, U = np.linalg.eig(F)
    en = np.angle(ev) / (2 * math.pi)
    p = np.argsort(en, kind="stable")
    return en[p], U[:, p]


def wilson_slices(h, NX, NY, bands, direction=1):
    """WilsonSlice1D of Wilson2D (Spectrum/berry.jl:258-268,340-367) on the periodic grid of the
    first NX-1 x NY-1 points: direction 1 one loop along j per i, direction 2 along i per j."""
    S = statesgrid(h, NX, NY, bands)[: NX - 1, : NY - 1]
    if direction == 2:
        S = np.transpose(S, (1, 0, 2, 3))
    en, Us = [], []
    for i in range(S.shape[0]):
        e, U = wilson1d(S[i])
        en.append(e)
        Us.append(U)
    return np.array(en), np.array(Us)


def wilson1d_base(grid3, j0):
    """Wilson1D(statesgrid, j0) (Spectrum/berry.jl:312-327) with the loop started at point j0."""
    NY = grid3.shape[0]
    return wilson1d(np.roll(grid3, -j0, axis=0))


def _abelian_loop(grid2):
    # Wilson1D(statesgrid (NY, M1)) (Spectrum/berry.jl:329-338)
    F = 1.0 + 0j
    for j in range(grid2.shape[0]):
        F *= np.vdot(grid2[j], grid2[(j + 1) % grid2.shape[0]])
    return np.angle(F) / (2 * math.pi)


def wilson_wannier2d(h, NX, NY, bands):
    """WilsonWannier2D(H, NX, NY, bandindices) (Spectrum/berry.jl:274-301): the states rotated
    by the eigenvectors of the loops through each point (Wilson1D with that base point),
    then per band the mean over the other direction's abelian Wilson loops: (p1, p2)."""
    S = statesgrid(h, NX, NY, bands)[: NX - 1, : NY - 1]
    nx, ny, _, m = S.shape
    new1 = np.empty_like(S)
    for i in range(nx):
        for j in range(ny):
            _, U = wilson1d_base(S[i, :, :, :], j)
            new1[i, j] = S[i, j] @ U
    new2 = np.empty_like(S)
    for i in range(nx):
        for j in range(ny):
            _, U = wilson1d_base(S[:, j, :, :], i)
            new2[i, j] = S[i, j] @ U
    p1 = [float(np.mean([_abelian_loop(new1[:, j, :, q]) for j in range(ny)])) for q in range(m)]
    p2 = [float(np.mean([_abelian_loop(new2[i, :, :, q]) for i in range(nx)])) for q in range(m)]
    return p1, p2


def fermidirac(e, mu=0.0, T=0.0):
    """Utils/fermidirac.jl:1-5: 1/(exp((e-mu)/T)+1) for T>0, else Heaviside(mu-e)
    with value 0.5 at equality."""
    x = np.asarray(e, float) - mu
    if T > 0:
        with np.errstate(over="ignore"):
            return 1.0 / (np.exp(x / T) + 1.0)
    return np.where(-x < 0, 0.0, np.where(-x > 0, 1.0, 0.5))


def chemicalpotential_0(energies, filling):
    """Spectrum/chemicalpotential.jl:9-23."""
    en = np.array(energies, float).ravel()
    if filling >= 1.0:
        return float(en.max())
    if filling <= 0.0:
        return float(en.min() - 1.0)
    i = 1 + int(math.floor(filling * (len(en) - 1)))  # 1-based
    s = np.sort(en)
    return float((s[i - 1] + s[i]) / 2)


def _f2u(x):
    return struct.unpack("<Q", struct.pack("<d", abs(x)))[0]


def _u2f(u):
    return struct.unpack("<d", struct.pack("<Q", u))[0]


def float_midpoint(a, b):
    """Midpoint over the float64 total order, as Roots.jl v2's Bisection uses:
    0.0 when the ends straddle zero, else the mean of the bit patterns of |a|,|b|
    carrying their common sign."""
    if (a < 0 < b) or (b < 0 < a):
        return 0.0
    m = _u2f((_f2u(a) + _f2u(b)) >> 1)
    return -m if (a + b) < 0 else m


def bisect_float(g, a, b, maxiter=200):
    """Bracketing bisection to adjacent floats (Roots.jl v2 ``Bisection``, the
    default of ``find_zero(f, (a, b))`` called at Spectrum/chemicalpotential.jl:37;
    Roots is not vendored in the reference, this restates its published algorithm).
    Returns the root to within one ulp."""
    fa, fb = g(a), g(b)
    if fa == 0:
        return a
    if fb == 0:
        return b
    if np.sign(fa) == np.sign(fb):
        raise ValueError("bracket does not change sign")
    for _ in range(maxiter):
        m = float_midpoint(a, b)
        if m == a or m == b:
            break
        fm = g(m)
        if fm == 0:
            return m
        if np.sign(fm) == np.sign(fa):
            a, fa = m, fm
        else:
            b, fb = m, fm
    return a if abs(fa) <= abs(fb) else b


def getfilling(bands, mu, T, weights=None):
    """Spectrum/chemicalpotential.jl:74-78: unweighted mean of f over all levels,
    or sum_k w_k sum_n f / n_bands with weights."""
    f = fermidirac(bands, mu, T)
    if weights is None:
        return float(np.mean(f))
    return float(np.sum(np.asarray(weights)[None, :] * f) / bands.shape[0])


def chemicalpotential(bands, filling, T=0.0, weights=None):
    """Spectrum/chemicalpotential.jl:6,32-38."""
    if T == 0:
        return chemicalpotential_0(bands, filling)
    g = lambda mu: getfilling(bands, mu, T, weights) - filling
    return bisect_float(g, float(bands.min()), float(bands.max()))


def densitymatrix(h, ks, w, mu, T, Lkeys, return_parts=False):
    """rho_L = sum_k w_k exp(-i 2 pi k.L) U f U^dagger and band energy sum_k w_k sum f eps.

    Operators/densitymatrix.jl:28-49 (driver) and :130-145 (per-k kernel)."""
    n = next(iter(h.values())).shape[0]
    rho = {L: np.zeros((n, n), complex) for L in Lkeys}
    eband = 0.0
    for j in range(ks.shape[1]):
        k = ks[:, j]
        e, U = eigh_upper(fouriersum(h, k), True)
        f = fermidirac(e, mu, T)
        rk = (U * f[None, :]) @ U.conj().T
        for L in Lkeys:
            rho[L] += w[j] * np.exp(-1j * 2 * math.pi * float(np.dot(k, np.array(L, float)))) * rk
        eband += float(np.real(w[j] * np.sum(e * f)))
    return rho, eband


def select_window(e, num_bands, sigma=1e-8, which="LM"):
    """Indices of the eigenpairs eigen_sparse returns (Eigen/eigen_sparse_krylovkit.jl:44-88),
    ascending: the num_bands eigenvalues nearest sigma (:LM; shift-invert Lanczos
    converged to its 1e-12 tolerance returns exactly those), the smallest (:SR) or the
    largest (:LR).  On a tie in distance the lower eigenvalue is taken (KrylovKit leaves
    ties unspecified; the reference's default sigma = 1e-8 avoids the symmetric ones)."""
    n = len(e)
    which = str(which).lstrip(":")
    if which == "SR":
        return np.arange(num_bands)
    if which == "LR":
        return np.arange(n - num_bands, n)
    order = sorted(range(n), key=lambda i: (abs(e[i] - sigma), e[i]))
    return np.sort(np.array(order[:num_bands]))


def bandmatrix_partial(h, ks, num_bands, sigma=1e-8, which="LM", vectors=False):
    """bandmatrix(H, ks; format=:sparse, num_bands) (Spectrum/bands.jl:78-87 with
    Eigen/Eigen.jl:35-39): bands (num_bands, nk), optionally U (nk, n, num_bands)."""
    n = next(iter(h.values())).shape[0]
    nk = ks.shape[1]
    bands = np.zeros((num_bands, nk))
    U = np.zeros((nk, n, num_bands), complex) if vectors else None
    for j in range(nk):
        e, u = eigh_upper(fouriersum(h, ks[:, j]), True)
        idx = select_window(e, num_bands, sigma, which)
        bands[:, j] = e[idx]
        if vectors:
            U[j] = u[:, idx]
    return bands, U


def densitymatrix_partial(h, ks, w, mu, T, Lkeys, num_bands, sigma=1e-8, which="LM"):
    """getdensitymatrix! with format=:sparse (Operators/densitymatrix.jl:100-104,131-147):
    rho_k = U_w f U_w^dagger over the selected states only."""
    n = next(iter(h.values())).shape[0]
    rho = {L: np.zeros((n, n), complex) for L in Lkeys}
    eband = 0.0
    for j in range(ks.shape[1]):
        k = ks[:, j]
        e, U = eigh_upper(fouriersum(h, k), True)
        idx = select_window(e, num_bands, sigma, which)
        e, U = e[idx], U[:, idx]
        f = fermidirac(e, mu, T)
        rk = (U * f[None, :]) @ U.conj().T
        for L in Lkeys:
            rho[L] += w[j] * np.exp(-1j * 2 * math.pi * float(np.dot(k, np.array(L, float)))) * rk
        eband += float(np.real(w[j] * np.sum(e * f)))
    return rho, eband


def dos(h, ks, omegas, gamma, w=None):
    """DOS(w) = sum_k w_k sum_n Im[1/(w - i Gamma - eps)], /L when unweighted.
    Spectrum/dos.jl:185-188 (dos!) and :202-223 (dos_compute!)."""
    omegas = np.asarray(omegas, float)
    out = np.zeros_like(omegas)
    for j in range(ks.shape[1]):
        e = eigh_upper(fouriersum(h, ks[:, j]), False)
        wt = 1.0 if w is None else w[j]
        out += np.sum(np.imag(wt * 1.0 / (omegas[:, None] - 1j * gamma - e[None, :])), axis=1)
    if w is None:
        out /= ks.shape[1]
    return out


def dos_from_bands(bands, omegas, gamma, w=None):
    """Same Lorentzian sum from precomputed bands (n, nk)."""
    omegas = np.asarray(omegas, float)
    nk = bands.shape[1]
    wt = np.ones(nk) if w is None else np.asarray(w, float)
    out = np.zeros_like(omegas)
    for j in range(nk):
        out += np.sum(np.imag(wt[j] / (omegas[:, None] - 1j * gamma - bands[None, :, j])), axis=1)
    if w is None:
        out /= nk
    return out
