"""Hopping models (Hops) restated from LatticeQM.jl (input construction for the workloads).

A Hops is a Python dict ``{R (tuple of ints): ndarray (n, n) complex128}``,
the restatement of ``Hops{K,T}`` (src/modules/TightBinding/types.jl:54-56).
Dict insertion order is the summation order of the Bloch sum.
"""
import math
import numpy as np

from . import lattice as L

SQRT_EPS = math.sqrt(np.finfo(float).eps)
SIGMA0 = np.eye(2, dtype=complex)
SIGMAX = np.array([[0, 1], [1, 0]], dtype=complex)
SIGMAY = np.array([[0, -1j], [1j, 0]], dtype=complex)
SIGMAZ = np.array([[1, 0], [0, -1]], dtype=complex)


def hopdim(h):
    return next(iter(h.values())).shape[0]


def zerokey(h):
    return tuple(0 for _ in next(iter(h.keys())))


def neighbor_dict(lat, cellrange):
    # Operators/gethops.jl:58-62 -> Lattices/neighbors.jl:153-165
    cells = L.getneighborcells(lat.A, cellrange, halfspace=True, innerpoints=True,
                               excludeorigin=False)
    nall = 3 + lat.extra.shape[0]
    out = {}
    for c in cells:
        da = np.zeros(nall)
        da[:3] = lat.A @ np.array(c, float)
        out[c] = da
    return out


def trim(h):
    # TightBinding/types.jl:278-286: drop blocks that are exactly zero
    return {R: M for R, M in h.items() if np.any(M != 0)}


def gethops_scalar(lat, t, cellrange=2, precision=SQRT_EPS):
    """Non-vectorized ``hops!``/``hoppingmatrix!`` (gethops.jl:86-140)."""
    Rpos = lat.allpositions()
    h = {}
    for dL, da in neighbor_dict(lat, cellrange).items():
        Ri = Rpos + da[:, None]
        N = Rpos.shape[1]
        M = np.zeros((N, N), dtype=complex)
        for i in range(N):
            for j in range(N):
                v = t(Ri[:, i], Rpos[:, j])
                if abs(v) >= precision:
                    M[i, j] = v
        h[dL] = M
        if any(x != 0 for x in dL):
            h[tuple(-x for x in dL)] = M.conj().T.copy()
    return trim(h)


def distance_window(a=1.0, halfwidth=0.01, t0=-1.0):
    # Operators/nearestneighbor.jl:22-47 (DistanceWindowHopping, 3-D spatial norm)
    def t(r1, r2):
        r = float(np.linalg.norm(r1[:3] - r2[:3]))
        return t0 if (a + halfwidth > r > a - halfwidth) else 0.0
    return t


def nearestneighbor(lat, t0=-1.0, a=1.0, halfwidth=0.01, cellrange=2):
    # Operators/nearestneighbor.jl:60-62
    return gethops_scalar(lat, distance_window(a, halfwidth, t0), cellrange=cellrange)


def graphene_block(R1, R2, tmin=1e-5, tz=0.46, t0=1.0, linter=0.125, lintra=0.08, z=3.0,
                   a=1.0, dmin=0.1, dmax=5.0):
    """``addgraphenematrix!`` (Operators/graphene.jl:242-274): out[i,j] = t(R1[:,i]-R2[:,j])."""
    d = R1[:3, :, None] - R2[:3, None, :]
    D = np.sqrt((d * d).sum(axis=0))
    with np.errstate(divide="ignore", invalid="ignore"):
        chi = d[2] ** 2 / D ** 2
        v = -t0 * (1 - chi) * np.exp(-np.abs(D - a) / lintra) \
            - tz * chi * np.exp(-np.abs(D - z) / linter)
    keep = (D <= dmax) & (D >= dmin) & (np.abs(v) >= tmin)
    return np.where(keep, v, 0.0).astype(complex)


def graphene(lat, cellrange=2, spin=False, **kw):
    """``Operators.graphene`` vectorized path (graphene.jl:17-28, gethops.jl:111-124)."""
    Rpos = lat.allpositions()
    h = {}
    for dL, da in neighbor_dict(lat, cellrange).items():
        M = graphene_block(Rpos + da[:, None], Rpos, **kw)
        h[dL] = M
        if any(x != 0 for x in dL):
            h[tuple(-x for x in dL)] = M.conj().T.copy()
    h = trim(h)
    return addspin(h) if spin else h


def addspin(h, mode="spinhalf"):
    # TightBinding/types.jl:258-270: kron(H, sigma), spin is the fast index
    s = {"spinhalf": SIGMA0, "σ0": SIGMA0, "σx": SIGMAX}[mode]
    return {R: np.kron(M, s) for R, M in h.items()}


def hermitianize(h):
    # TightBinding/types.jl:174-189
    for R in list(h.keys()):
        mR = tuple(-x for x in R)
        if mR in h:
            h[R] = (h[R] + h[mR].conj().T) / 2
            h[mR] = h[R].conj().T.copy()
        else:
            h[mR] = h[R].conj().T.copy()
    return h


def currentoperators(lat, h):
    """``getcurrentoperators(lat, hops)`` (Operators/current.jl:20-37 with
    _apply_position_factor_dense!, :65-75): one Hops per lattice direction alpha,
    J_alpha[R] = H_R with block (i, j) (orbital pair, size D/N for the internal
    multiplicity) multiplied by -i (r_i + A R - r_j)_alpha, r the Cartesian
    positions, alpha the Cartesian component."""
    r = lat.positions()
    A = lat.basis[:, :2]
    N = r.shape[1]
    D = hopdim(h)
    if D < N or D % N:
        raise ValueError("Hops dimension is not a multiple of the orbital count")
    m = D // N
    Js = []
    for a in range(A.shape[1]):
        J = {}
        for R, M in h.items():
            r0 = r[a] + (A @ np.array(R, float))[a]
            fac = -1j * (r0[:, None] - r[a][None, :])  # (i, j) -> -i (r0_i - r_j)
            J[R] = M * np.kron(fac, np.ones((m, m)))
        Js.append(J)
    return Js


def with_keys(h, keys):
    """Restrict/extend a Hops to exactly ``keys`` (zero blocks kept)."""
    n = hopdim(h)
    for R, M in h.items():
        if R not in keys and np.any(M != 0):
            raise ValueError(f"nonzero block {R} outside the requested key set")
    return {R: (h[R].copy() if R in h else np.zeros((n, n), complex)) for R in keys}


KEYS9 = [R for R in L.product_first_fastest(range(-1, 2), range(-1, 2))]


# --------------------------------------------------------------------------------------
# Workload builders (seeded synthetic inputs of the named shapes)
# --------------------------------------------------------------------------------------

def honeycomb_disorder(L_super=6, sigma=0.1, seed=1):
    """Spinful honeycomb NN model, t=-1, L_super x L_super supercell, onsite disorder
    N(0, sigma) equal on both spins; keys = the 9 vectors of {-1,0,1}^2 (zero blocks kept).
    n = 4 * L_super^2 (144 for the 6x6 cell)."""
    lat = L.superlattice(L.honeycomb(), [L_super, L_super])
    h = nearestneighbor(lat, -1.0)
    h = with_keys(addspin(h), KEYS9)
    rng = np.random.default_rng(seed)
    eps = rng.normal(0.0, sigma, lat.norb)
    h[(0, 0)] += np.diag(np.repeat(eps, 2)).astype(complex)
    return lat, h


def _shell_distances(lat, nshell):
    pos = lat.positions()
    ds = set()
    for c in L.product_first_fastest(range(-2, 3), range(-2, 3)):
        da = lat.A @ np.array(c, float)
        d = np.linalg.norm(pos[:, :, None] + da[:, None, None] - pos[:, None, :], axis=0)
        ds.update(np.round(d[d > 1e-9], 9).ravel().tolist())
    return sorted(ds)[:nshell]


def random_bonds(lat, rng, nshell=2, tdist=(-1.0, 1.0), onsite_sigma=0.2, soc=False):
    """Random real NN+NNN hoppings t~U(tdist) per bond plus onsite N(0, onsite_sigma),
    spinful.  With ``soc`` each bond carries a spin-orbit phase exp(i phi sigma_z),
    phi~U(0, 2pi).  The Hermitian partner H_{-R} = H_R^dagger is set per bond
    (the role of ``hermitianize!``, TightBinding/types.jl:174-189)."""
    shells = _shell_distances(lat, nshell)
    pos = lat.positions()
    N = lat.norb
    blocks = {R: np.zeros((2 * N, 2 * N), complex) for R in KEYS9}
    for R in KEYS9:
        mR = tuple(-x for x in R)
        if R > mR:
            continue  # handle each +/-R pair once (R == mR only for R = 0)
        da = lat.A @ np.array(R, float)
        for i in range(N):
            for j in range(N):
                if R == mR and j <= i:
                    continue
                dd = round(float(np.linalg.norm(pos[:, i] + da - pos[:, j])), 9)
                if not any(abs(dd - s) < 1e-6 for s in shells):
                    continue
                t = rng.uniform(*tdist)
                if soc:
                    phi = rng.uniform(0.0, 2 * math.pi)
                    blk = t * np.diag([np.exp(1j * phi), np.exp(-1j * phi)])
                else:
                    blk = t * SIGMA0
                blocks[R][2 * i:2 * i + 2, 2 * j:2 * j + 2] += blk
                blocks[mR][2 * j:2 * j + 2, 2 * i:2 * i + 2] += blk.conj().T
    eps = rng.normal(0.0, onsite_sigma, N)
    blocks[(0, 0)] += np.diag(np.repeat(eps, 2))
    return blocks


def batch_models(seed=2):
    """The three uneven models of the batched workload: square 2x2 (n=8), kagome 2x2
    (n=24) and triangular 4x4 with spin-orbit phases (n=96: 4x4 copies of the 3-site
    ``triangular_supercell`` cell, 2d.jl:87-93, spinful)."""
    rng = np.random.default_rng(seed)
    out = []
    sq = L.superlattice(L.square(), [2, 2])
    out.append(("square2x2", random_bonds(sq, rng)))
    kg = L.superlattice(L.kagome(), [2, 2])
    out.append(("kagome2x2", random_bonds(kg, rng)))
    tr = L.superlattice(L.triangular_supercell(), [4, 4])
    out.append(("triangular4x4_soc", random_bonds(tr, rng, soc=True)))
    return out


def hubbard_v(lat, U=4.0, a=0.5, mode="σx", neighbors=((0, 0),)):
    """``gethubbard(lat, neighbors; mode, a, U)`` (Operators/interactions.jl:8,18-28):
    for each cell offset dL in ``neighbors`` the block V_dL[i, j] = U * heaviside(a - r),
    r = |r_i + A dL - r_j| (heaviside(0) = 1/2), and for dL != 0 its Hermitian partner
    V_{-dL} = V_dL^H (Operators/gethops.jl:96-109, ``hops[-δL] = hops[δL]'``, so a
    one-sided neighbour list still gives a Hermitian V); all-zero blocks are dropped
    (``trim!``, TightBinding/types.jl:278-285); then spin added in ``mode`` (σx: the
    kron with sigma_x)."""
    N = lat.norb
    pos = lat.allpositions()
    out = {}
    for dL in neighbors:
        dL = tuple(int(x) for x in dL)
        shift = lat.A @ np.array(dL, float)
        V = np.zeros((N, N), complex)
        for i in range(N):
            for j in range(N):
                r = float(np.linalg.norm(pos[:3, i] + shift - pos[:3, j]))
                v = U * (0.0 if a - r < 0 else (1.0 if a - r > 0 else 0.5))
                if abs(v) >= SQRT_EPS:
                    V[i, j] = v
        out[dL] = V
        if any(x != 0 for x in dL):
            out[tuple(-x for x in dL)] = V.conj().T.copy()
    out = {dL: V for dL, V in out.items() if np.any(V != 0)}
    return addspin(out, mode)


def triangular_hubbard(L_super=6, t=-1.0, tp=0.2, U=4.0):
    """Spinful triangular-lattice Hubbard model on an L x L supercell (n = 2 L^2):
    NN hopping t, NNN hopping tp, v = Hubbard(U) in the sigma_x mode."""
    lat = L.superlattice(L.triangular(), [L_super, L_super])
    h1 = nearestneighbor(lat, t, a=1.0)
    h2 = nearestneighbor(lat, tp, a=math.sqrt(3.0))
    h = {}
    for hh in (h1, h2):
        for R, M in hh.items():
            h[R] = h.get(R, 0) + M
    h = addspin(h)
    v = hubbard_v(lat, U=U)
    return lat, h, v


def nn_bond_length(lat):
    """The shortest nonzero distance between orbitals of neighbouring cells
    (Operators/haldane.jl, _nnbondlength)."""
    pos = lat.positions()
    d = math.inf
    for c in L.product_first_fastest(range(-1, 2), range(-1, 2)):
        sh = lat.A @ np.array(c, float)
        dist = np.linalg.norm(pos[:, :, None] + sh[:, None, None] - pos[:, None, :], axis=0)
        nz = dist[dist > SQRT_EPS]
        if nz.size:
            d = min(d, float(nz.min()))
    return d


def add_haldane(h, lat, t2, phi=math.pi / 2, cellrange=1):
    """``addhaldane!(hops, lat, t2; ϕ)`` (Operators/haldane.jl, naive path): for every pair
    (i in cell R, j in cell 0) at distance sqrt(3) a0, with R0 their first common nearest
    neighbour found over the cells {-1..1}^2 and the orbitals, x = r_i + A R - R0,
    y = r_j - R0: h[R][i, j] += t2 exp(i phi sign(cross(-y, x))).  Returns a new dict."""
    pos = lat.positions()
    N = lat.norb
    a0 = nn_bond_length(lat)
    cells = L.product_first_fastest(range(-cellrange, cellrange + 1), range(-cellrange, cellrange + 1))
    near = L.product_first_fastest(range(-1, 2), range(-1, 2))
    out = {R: M.copy() for R, M in h.items()}
    cross = lambda x, y: x[0] * y[1] - x[1] * y[0]
    for R in cells:
        sh = lat.A @ np.array(R, float)
        for i in range(N):
            for j in range(N):
                ri, rj = pos[:, i] + sh, pos[:, j]
                if not math.isclose(float(np.linalg.norm(ri - rj)), math.sqrt(3) * a0, rel_tol=1e-6):
                    continue
                found = None
                for c in near:
                    dc = lat.A @ np.array(c, float)
                    for m in range(N):
                        r0 = dc + pos[:, m]
                        if (math.isclose(float(np.linalg.norm(ri - r0)), a0, rel_tol=1e-6)
                                and math.isclose(float(np.linalg.norm(rj - r0)), a0, rel_tol=1e-6)):
                            found = r0
                            break
                    if found is not None:
                        break
                if found is None:
                    continue
                x, y = ri - found, rj - found
                if R not in out:
                    out[R] = np.zeros((N, N), complex)
                out[R][i, j] += t2 * np.exp(1j * phi * np.sign(cross(-y, x)))
    return out


def haldane_model(t1=-1.0, t2=0.1, phi=math.pi / 2):
    """Honeycomb nearest-neighbour model t1 with the Haldane term t2 e^{±i phi}
    (the model of test/test_haldane.jl)."""
    lat = L.honeycomb()
    return lat, add_haldane(nearestneighbor(lat, t1), lat, t2, phi)


def bdg_operator(h, delta=None):
    """``BdGOperator(h[, Δ])`` (Superconductivity/types.jl:43-60,76-97): the Nambu Hops of
    order 2d with blocks [h_R 0; 0 -conj(h_R)] and, for every pairing key R (its partner
    -R present), [0 Δ_R; Δ_{-R}^H 0]."""
    d = hopdim(h)
    H = {}
    for R, M in h.items():
        B = np.zeros((2 * d, 2 * d), complex)
        B[:d, :d] = M
        B[d:, d:] = -np.conj(M)
        H[R] = B
    for R, D in (delta or {}).items():
        mR = tuple(-x for x in R)
        if mR not in delta:
            raise ValueError(f"pairing key {R} has no partner {mR}")
        B = np.zeros((2 * d, 2 * d), complex)
        B[:d, d:] = D
        B[d:, :d] = np.asarray(delta[mR]).conj().T
        H[R] = H[R] + B if R in H else B
    return H


def antiferro_density(lat):
    """``initialguess(v, :antiferro; lat)`` (Meanfield/initialguess.jl:186-193):
    rho_0 = kron(P_A, rho_up) + kron(P_B, sigma0 - rho_up), rho_up = diag(1, 0), P_A/P_B the
    projectors on sublattice 0/1 (spin the fast index)."""
    sub = lat.extracoord("sublattice")
    up = np.diag([1.0, 0.0]).astype(complex)
    PA = np.diag((sub == 0).astype(float))
    PB = np.diag((sub == 1).astype(float))
    return np.kron(PA, up) + np.kron(PB, SIGMA0 - up)


def graphene_hubbard(U=4.0):
    """The commutator-residual SCF case of test/test_meanfield.jl:84-112: spinful
    ``Operators.graphene`` on the honeycomb cell, Hubbard v (mode sigma_x, a = 0.5, U)
    and the antiferromagnetic initial guess (n = 4)."""
    lat = L.honeycomb()
    h = graphene(lat, spin=True)
    v = hubbard_v(lat, U=U, a=0.5)
    return lat, h, v, {(0, 0): antiferro_density(lat)}


def random_local_magnetization(n_sites, seed=3):
    """Seeded ``mapspindensitymatrix(:random, n)`` (Meanfield/initialguess.jl:24-35,48-58,
    68-80): per site 1/2 (sigma0 + d.sigma) with a random unit vector d."""
    rng = np.random.default_rng(seed)
    M = np.zeros((2 * n_sites, 2 * n_sites), complex)
    for i in range(n_sites):
        th = math.pi * rng.random()
        ph = 2 * math.pi * rng.random()
        d = [math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)]
        M[2 * i:2 * i + 2, 2 * i:2 * i + 2] = 0.5 * (SIGMA0 + d[0] * SIGMAX + d[1] * SIGMAY
                                                      + d[2] * SIGMAZ)
    return M


def tbg_slater_koster(N, **kw):
    """Twisted bilayer (m=N, r=1) with the Slater-Koster parameters of the precision
    workload: Vppπ=-2.7, Vppσ=+0.48, decay 0.184*a_lat (a_lat = sqrt(3) NN distances),
    cutoff 3*a_lat; spinless, n = 4 (3N^2+3N+1)."""
    lat = L.honeycomb_twisted(N)
    dlt = 0.184 * math.sqrt(3.0)
    params = dict(t0=2.7, tz=-0.48, lintra=dlt, linter=dlt, a=1.0, z=3.0,
                  dmax=3 * math.sqrt(3.0), tmin=1e-5)
    params.update(kw)
    return lat, graphene(lat, **params)


def screened_coulomb_v(lat, V0=1.4 * math.sqrt(3.0), lam=10.0 * math.sqrt(3.0), onsite=1.4, cellrange=1):
    """Density-density interaction v_R[i, j] = V0 exp(-d/lam) / d with d = |r_i + R - r_j|
    (``Hops(lat, V; cellrange)``, gethops.jl:33-36, with V(r) = V0 e^{-r/lam}/r), the
    divergent d = 0 entries replaced by ``onsite``.  Defaults: the large twisted-bilayer
    workload, V0 = 1.4 eV * a and lam = 10 a with a = sqrt(3) (graphene lattice constant
    in units of the nearest-neighbour distance) and the cap V0 / a = 1.4 eV on site."""
    Rpos = lat.allpositions()
    v = {}
    for dL, da in neighbor_dict(lat, cellrange).items():
        R1 = Rpos + da[:, None]
        d = R1[:3, :, None] - Rpos[:3, None, :]
        D = np.sqrt((d * d).sum(axis=0))
        with np.errstate(divide="ignore", invalid="ignore"):
            M = np.where(D > 1e-9, V0 * np.exp(-D / lam) / D, onsite)
        v[dL] = M.astype(complex)
        if any(x != 0 for x in dL):
            v[tuple(-x for x in dL)] = v[dL].T.copy()
    return v


def tbg_screened_hf(N):
    """Twisted bilayer (m=N, r=1) Slater-Koster hopping with the screened Coulomb
    interaction of the large Hartree-Fock workload: (lat, h, v)."""
    lat, h = tbg_slater_koster(N)
    return lat, h, screened_coulomb_v(lat)
