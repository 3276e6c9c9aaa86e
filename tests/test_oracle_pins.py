"""Pin the CPU oracle to the reference's own golden vectors and known answers.

Sources (LatticeQM.jl): test/analyticbands.jl:5-16 with test/test_spectrum_graphene.jl:15-30,
test/test_spectrum_square.jl:10-35, test/test_spectrum_triangular.jl:10-33,
test/test_tbg.jl:52-94,213-257 (values extracted to tests/golden/reference_pins.json),
test/test_spectrum_graphene.jl:42-63 (DOS invariants), test/test_meanfield.jl:228-278
(HF variational identity).
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import kspace as K
from lqm_workloads import lattice as L
from oracle import meanfield as MF
from lqm_workloads import models as M

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def graphene_conduction(k):
    # test/analyticbands.jl:5-16
    rs = [[1, 0], [-1, 0], [0, 1], [0, -1], [1, -1], [-1, 1]]
    return math.sqrt(3.0 + sum(math.cos(2 * math.pi * np.dot(k, r)) for r in rs))


def pin_index(expr, n):
    expr = expr.replace(" ", "")
    table = {"end": n - 1, "end-1": n - 2, "end÷2": n // 2 - 1, "end÷2+1": n // 2}
    return table[expr] if expr in table else int(expr) - 1


def test_graphene_nn_bands_analytic():
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    ks = L.kpath(lat, 200)
    b, _ = K.bandmatrix(h, ks)
    up = np.array([graphene_conduction(k) for k in ks.T])
    assert np.sum(np.abs(b[0] + up)) + np.sum(np.abs(b[1] - up)) < 1e-12


def test_square_nn_bands_analytic():
    lat = L.square()
    h = M.nearestneighbor(lat, -1.0)
    ks = L.kpath(lat, 200)
    b, _ = K.bandmatrix(h, ks)
    ana = -2 * (np.cos(2 * np.pi * ks[0]) + np.cos(2 * np.pi * ks[1]))
    assert np.max(np.abs(b[0] - ana)) < 1e-12


def test_triangular_nn_bands_analytic():
    lat = L.triangular()
    h = M.nearestneighbor(lat, -1.0)
    ks = L.kpath(lat, 200)
    b, _ = K.bandmatrix(h, ks)
    ana = -2 * (np.cos(2 * np.pi * ks[0]) + np.cos(2 * np.pi * ks[1]) + np.cos(2 * np.pi * (ks[0] - ks[1])))
    assert np.max(np.abs(b[0] - ana)) < 1e-12


def test_tbg_lattice_fixture():
    # test/test_tbg.jl:19-49
    lat = L.honeycomb_twisted(1)
    assert lat.norb == 28
    layer = lat.extracoord("layer")
    assert np.sum(layer == 0) == 14 and np.sum(layer == 1) == 14
    A = lat.A
    assert abs(np.linalg.norm(A[:, 0]) - math.sqrt(21)) < 1e-12
    assert abs(L.twistangle(1) - math.acos(6.5 / 7)) < 1e-14
    assert np.array_equal(L.moire_supercell(1, 1), np.array([[1, -2], [2, 3]]))


_BUILDERS = {"honeycomb_twisted": L.honeycomb_twisted, "honeycomb_twisted_ABBA": L.honeycomb_twisted_ABBA,
             "honeycomb_twisted_ABAB": L.honeycomb_twisted_ABAB}


def test_tbg_eigenvalue_pins():
    pins = json.load(open(os.path.join(GOLD, "reference_pins.json")))["pins"]
    cache = {}
    for p in pins:
        key = (p["builder"], p["N"])
        if key not in cache:
            cache[key] = M.graphene(_BUILDERS[p["builder"]](p["N"]), tz=0.32)
        h = cache[key]
        ev = K.eigh_upper(K.fouriersum(h, p["k"]), vectors=False)
        i = pin_index(p["index"], len(ev))
        assert abs(ev[i] - p["value"]) <= p["atol"], p


def test_tbg_near_degenerate_pair_at_K():
    # test/test_tbg.jl:90-92
    h = M.graphene(L.honeycomb_twisted(1), tz=0.32)
    ev = K.eigh_upper(K.fouriersum(h, [1 / 3, -1 / 3]), vectors=False)
    assert abs(ev[13] - ev[12]) < 1e-12 and abs(ev[14] - ev[15]) < 1e-12


def test_graphene_dos_invariants():
    # test/test_spectrum_graphene.jl:42-63 on a 60x60 grid (the test uses 120x120)
    h = M.nearestneighbor(L.honeycomb(), -1.0)
    om = np.linspace(-3.05, 3.05, 401)
    ks = L.regulargrid(60 * 60)
    b, _ = K.bandmatrix(h, ks)
    dos = K.dos_from_bands(b, om, 0.05)
    assert np.max(np.abs(dos - dos[::-1])) / np.max(np.abs(dos)) < 1e-10
    assert abs(np.sum(dos) * (om[1] - om[0]) - 2 * math.pi) / (2 * math.pi) < 0.05
    i0, ip, im = np.argmin(np.abs(om)), np.argmin(np.abs(om - 1)), np.argmin(np.abs(om + 1))
    assert dos[ip] > 3 * dos[i0] and dos[im] > 3 * dos[i0]


def test_densitymatrix_band_energy_matches_direct():
    # test/test_operators.jl:91-128: getdensitymatrix! band energy == sum_k tr(rho_k H_k)/L
    h = M.graphene(L.honeycomb(), spin=True)
    nk = 9
    ks = np.array([[i / nk, j / nk] for j in range(nk) for i in range(nk)]).T
    mu = -0.5
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    rho, eb = K.densitymatrix(h, ks, w, mu, 0.0, list(h.keys()))
    direct = 0.0
    for k in ks.T:
        Hk = K.fouriersum(h, k)
        e, U = np.linalg.eigh(Hk)
        rk = (U * (e < mu)) @ U.conj().T
        direct += np.real(np.trace(rk @ Hk))
    direct /= ks.shape[1]
    assert abs(eb - direct) < 1e-10
    # expval pairing sum_L tr[rho_L H_{-L}] gives the same band energy
    ev = sum(np.real(np.trace(rho[L] @ h[tuple(-x for x in L)])) for L in rho)
    assert abs(ev - direct) < 1e-10


def test_hf_variational_identity_complex_rho():
    # test/test_meanfield.jl:228-255
    lat = L.honeycomb()
    h = M.graphene(lat, spin=True)
    v = M.hubbard_v(lat, U=4.0)
    N = 4
    ii, jj = np.meshgrid(np.arange(1, N + 1), np.arange(1, N + 1), indexing="ij")
    Mm = np.exp(1j * (3 * ii + jj)) / (1 + np.abs(ii - jj))
    Mm = (Mm + Mm.conj().T) / 2
    rho = {(0, 0): Mm}
    hf = MF.HartreeFock(h, v)(rho)
    ks = np.array([[i / 3, j / 3] for j in range(3) for i in range(3)]).T

    def trprod(A, B):
        return sum(np.real(np.trace(K.fouriersum(A, k) @ K.fouriersum(B, k))) for k in ks.T) / ks.shape[1]

    assert abs(trprod(hf.hMF, rho) - trprod(h, rho) - 2 * (hf.eH + hf.eF)) < 1e-10


def test_float_bisection_reaches_adjacent_floats():
    g = lambda x: x ** 3 - 2.0
    r = K.bisect_float(g, 0.0, 3.0)
    assert abs(r - 2 ** (1 / 3)) <= 2 * np.spacing(2 ** (1 / 3))
    assert K.float_midpoint(-1.0, 2.0) == 0.0


def test_chemicalpotential_zero_T_order_statistics():
    # Spectrum/chemicalpotential.jl:9-23
    e = np.array([[0.0, 1.0, 2.0], [3.0, 4.0, 5.0]])
    assert K.chemicalpotential_0(e, 0.5) == 2.5
    assert K.chemicalpotential_0(e, 1.0) == 5.0
    assert K.chemicalpotential_0(e, 0.0) == -1.0


def test_regulargrid_order():
    ks = L.regulargrid(16)
    assert ks.shape == (2, 16)
    assert np.allclose(ks[:, 1], [0.25, 0.0]) and np.allclose(ks[:, 4], [0.0, 0.25])


@pytest.mark.parametrize("builder,n", [("honeycomb_disorder", 144), ("batch", None), ("hubbard", 72)])
def test_workload_shapes(builder, n):
    if builder == "honeycomb_disorder":
        _, h = M.honeycomb_disorder()
        assert M.hopdim(h) == n and len(h) == 9
    elif builder == "batch":
        assert [M.hopdim(h) for _, h in M.batch_models()] == [8, 24, 96]
    else:
        _, h, v = M.triangular_hubbard()
        assert M.hopdim(h) == n and list(v.keys()) == [(0, 0)]
    # Hermitian as Hops
    hh = h if builder != "batch" else M.batch_models()[2][1]
    for R, blk in hh.items():
        assert np.allclose(blk, hh[tuple(-x for x in R)].conj().T)


# ---------------------------------------------------------------- adjoints (finite differences)
def _small_model():
    from lqm_workloads import models as M
    return M.batch_models()[0][1]  # square 2x2 spinful, n = 8


def test_densitymatrix_vjp_matches_finite_differences():
    from oracle import adjoint as AD
    h = _small_model()
    rng = np.random.default_rng(4)
    ks = rng.random((2, 5))
    w = np.full(5, 0.2)
    mu, T = 0.1, 0.05
    keys = list(h.keys())
    Gbar = {L: rng.normal(size=h[L].shape) + 1j * rng.normal(size=h[L].shape) for L in keys}
    Hbar = AD.densitymatrix_vjp(h, ks, w, mu, T, Gbar)
    dH = AD.hermitian_direction(h, rng)

    def loss(hh):
        rho, _ = K.densitymatrix(hh, ks, w, mu, T, keys)
        return AD.pairing(Gbar, rho)

    step = 1e-6
    hp = {R: h[R] + step * dH[R] for R in h}
    hm = {R: h[R] - step * dH[R] for R in h}
    fd = (loss(hp) - loss(hm)) / (2 * step)
    an = AD.pairing(Hbar, dH)
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def test_bands_vjp_matches_finite_differences():
    from oracle import adjoint as AD
    h = _small_model()
    rng = np.random.default_rng(8)
    ks = rng.random((2, 4))
    n = h[(0, 0)].shape[0]
    # the spinful bands come in degenerate pairs: a loss that weights both members of
    # a pair alike is differentiable (the pair's projector is smooth)
    eb = np.repeat(rng.normal(size=(n // 2, ks.shape[1])), 2, axis=0)
    Hbar = AD.bands_vjp(h, ks, eb)
    dH = AD.hermitian_direction(h, rng)

    def loss(hh):
        return float(np.sum(eb * K.bandmatrix(hh, ks)[0]))

    step = 1e-6
    fd = (loss({R: h[R] + step * dH[R] for R in h}) - loss({R: h[R] - step * dH[R] for R in h})) / (2 * step)
    an = AD.pairing(Hbar, dH)
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def test_grand_potential_gradient_is_rho():
    """d/dH_R of -T sum_k w_k sum_j log(1 + exp(-(eps_j - mu)/T)) equals rho_R (Hellmann-Feynman)."""
    from oracle import adjoint as AD
    h = _small_model()
    rng = np.random.default_rng(9)
    ks = rng.random((2, 4))
    w = np.full(4, 0.25)
    mu, T = 0.0, 0.1
    keys = list(h.keys())
    rho, _ = K.densitymatrix(h, ks, w, mu, T, keys)
    dH = AD.hermitian_direction(h, rng)

    def omega(hh):
        b = K.bandmatrix(hh, ks)[0]
        return float(-T * np.sum(w * np.sum(np.logaddexp(0.0, -(b - mu) / T), axis=0)))

    step = 1e-6
    fd = (omega({R: h[R] + step * dH[R] for R in h}) - omega({R: h[R] - step * dH[R] for R in h})) / (2 * step)
    assert abs(fd - AD.pairing(rho, dH)) <= 1e-6 * max(1.0, abs(fd))


def test_band_expectation_values_known_answers():
    """bandmatrix(H, ks, projectors...) (bands.jl:52-60,107-112): with H itself as the
    projector the expectation values are the bands, with the identity they are 1, and
    graphene's sublattice polarisation vanishes away from the Dirac points."""
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    ks = L.kpath(lat, 64)
    n = h[(0, 0)].shape[0]
    sz = np.diag([1.0, -1.0]).astype(complex)
    bands, obs = K.bandmatrix_obs(h, ks, [h, np.eye(n), sz])
    assert np.max(np.abs(obs[:, :, 0] - bands)) < 1e-13
    assert np.max(np.abs(obs[:, :, 1] - 1.0)) < 1e-13
    gap = bands[1] - bands[0]
    away = gap > 1e-3
    assert np.max(np.abs(obs[:, away, 2])) < 1e-12


def test_anderson_scf_oracle_converges_faster_than_linear():
    """fixedpoint.jl's Anderson branch restated in the oracle: on the 2x2 Hubbard model it
    converges to 1e-10 in far fewer iterations than linear mixing, to the same energy (the
    magnetisation direction of the spin-rotation-invariant ground state may differ)."""
    lat, h, v = M.triangular_hubbard(L_super=2)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=3)}
    ks = L.regulargrid(6 * 6)
    a = MF.solvehartreefock(h, v, rho0, 0.5, ks, T=0.02, beta=0.3, tol=1e-10, iterations=200,
                            acceleration="anderson", anderson_depth=5)
    lin = MF.solvehartreefock(h, v, rho0, 0.5, ks, T=0.02, beta=0.3, tol=1e-10, iterations=2000)
    assert a[3] and lin[3]
    assert a[5] < lin[5] / 3
    assert abs(a[1] - lin[1]) < 1e-9


def test_density_and_ldos_sum_rules():
    """density (dos.jl:20-52): the orbital sum counts the states below mu per k-point;
    ldos (dos.jl:56-98): the orbital sum is the DOS over pi (the getdos normalisation
    has no 1/pi, dos.jl:138-144), for one frequency and for a window."""
    lat = L.honeycomb()
    h = M.graphene(lat, spin=True)
    ks = L.regulargrid(12 * 12)
    n = K.density(h, ks, mu=0.3)
    bands = K.bandmatrix(h, ks)[0]
    assert abs(n.sum() - np.mean(np.sum(bands <= 0.3, axis=0))) < 1e-12
    for om in ([0.4], [0.2, 0.5, 0.9]):
        ld = K.ldos(h, ks, om, gamma=0.05)
        dos = np.mean([K.dos_from_bands(bands, np.array([w]), 0.05)[0] for w in om])
        assert abs(ld.sum() - dos / np.pi) < 1e-12 * max(1.0, dos)


def test_berry_massive_graphene_valley_curvature():
    """berry.jl:107-155 restated: gapped graphene (staggered onsite) has zero total Chern
    number and opposite curvature at the two valleys (the plaquette phases sum to 0 and
    the grid's extreme values are negatives of each other)."""
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    h[(0, 0)] = h[(0, 0)] + np.diag([0.3, -0.3])
    F = K.berry(h, 12, 12, [0])
    assert abs(F.sum()) < 1e-12
    assert abs(F.max() + F.min()) < 1e-12 and F.max() > 0.05


def test_optical_conductivity_graphene_invariants():
    """test/test_linearresponse.jl:33-58 (graphene, half filling, klin=30, 30 frequencies:
    sigma_xx = sigma_yy, Re sigma_xy = 0, Re sigma_xx >= 0) and test/test_operators.jl:135-151
    (the current operators are Hermitian) on the oracle."""
    lat = L.honeycomb()
    h = M.graphene(lat)
    Js = M.currentoperators(lat, M.nearestneighbor(lat, -1.0))
    assert len(Js) == 2
    for k in ([0.0, 0.0], [1 / 3, -1 / 3], [0.5, 0.5], [-0.2, 0.7]):
        for J in Js:
            Jk = K.fouriersum(J, k)
            assert np.max(np.abs(Jk - Jk.conj().T)) < 1e-10
    Js = M.currentoperators(lat, h)
    om = np.linspace(0.05, 3.0, 30)
    gam, T, mu = 0.05, 0.01, 0.0
    ks = L.regulargrid(nk=30 ** 2)
    sig = {}
    for a, b in ((0, 0), (1, 1), (0, 1)):
        chi = K.opticalconductivity(om, h, Js[a], Js[b], ks, mu, gam, T)
        sig[a, b] = -(chi - chi[0]) / (om + 1j * gam)
    assert np.max(np.abs(sig[0, 0].real - sig[1, 1].real)) < 1e-10
    assert np.max(np.abs(sig[0, 1].real)) < 1e-10
    assert np.all(sig[0, 0].real > -1e-6)
    assert np.max(sig[0, 0].real) > 1e-3  # an interband response is present


def test_partial_spectrum_selection_rules():
    """test/test_eigen.jl:11-40,69-85 restated on the oracle's window selection: :LM at
    sigma=0 gives the num_bands eigenvalues of smallest modulus, :SR/:LR the ends of the
    spectrum, all ascending (a seeded 60 x 60 real symmetric matrix, entries U(-0.5, 0.5),
    stands in for the reference's Xoshiro draw)."""
    rng = np.random.default_rng(0x123456789ABCDEF)
    A = rng.random((60, 60)) - 0.5
    A = np.triu(A) + np.triu(A, 1).T
    h = {(0, 0): A.astype(complex)}
    ks = np.zeros((2, 1))
    e = np.sort(np.linalg.eigvalsh(A))
    lm, _ = K.bandmatrix_partial(h, ks, 10, sigma=0.0)
    assert np.allclose(lm[:, 0], np.sort(sorted(e, key=abs)[:10]), atol=1e-12)
    sr, _ = K.bandmatrix_partial(h, ks, 10, which="SR")
    lr, _ = K.bandmatrix_partial(h, ks, 10, which="LR")
    assert np.allclose(sr[:, 0], e[:10], atol=1e-12) and np.allclose(lr[:, 0], e[-10:], atol=1e-12)
    for which, sig in (("LM", 0.2), ("SR", 1e-8), ("LR", 1e-8)):
        b, U = K.bandmatrix_partial(h, ks, 6, sigma=sig, which=which, vectors=True)
        assert np.all(np.diff(b[:, 0]) >= 0)
        assert np.max(np.abs(A @ U[0] - U[0] * b[:, 0][None, :])) < 1e-10
    # a tie in distance takes the lower eigenvalue
    assert list(K.select_window(np.array([-1.0, 1.0, 3.0]), 1, sigma=0.0)) == [0]


def test_commutator_residual_scf_oracle():
    """test/test_meanfield.jl:84-112 (commutatorresidual) on the oracle: graphene Hubbard
    U = 4 from the antiferromagnetic guess, keys enriched to the klin = 9 Wigner-Seitz
    cell, Anderson depth 5, beta = 1, T = 0.01: converges below 1e-7 within 50 iterations
    and the commutator residual drops by more than 1e6."""
    _, h, v, rho0 = M.graphene_hubbard(4.0)
    MF.enrichkeys(rho0, 9)
    assert len(rho0) == 81
    ks = L.regulargrid(9 * 9)
    log = []
    rho, E, hf, conv, res, it = MF.solvehartreefock(
        h, v, rho0, 0.5, ks, T=0.01, beta=1.0, tol=1e-7, iterations=50, acceleration="anderson",
        anderson_depth=5, residual_norm="commutator", log=lambda i, e, r, *a: log.append(r))
    assert conv and res < 1e-7
    assert log[0] / log[-1] > 1e6
    # at the fixed point the commutator vanishes (the converged rho re-evaluated)
    hf(rho)
    assert MF.commutator_kspace_norm(hf.hMF, rho, ks) < 1e-6


def _jkernel(J1, Jnn):
    # test/test_exchange.jl:14-20: intra-cell J1 between sites 0-1, inter-cell site0-site0 Jnn
    j0 = np.array([[0.0, J1], [J1, 0.0]], complex)
    jp = np.array([[Jnn, 0.0], [0.0, 0.0]], complex)
    return {(0, 0): j0, (1, 0): jp, (-1, 0): jp.conj().T}


SITEOF0, FLAVOROF0 = [0, 1, 0, 1], [0, 0, 1, 1]  # flavor-outer layout of test_exchange.jl:11-12


def test_exchange_kernel_oracle_pins():
    """test/test_exchange.jl:29-83 on the oracle: construction rules, the analytic dimer
    limits (eJ = -J1 polarized, -J1/2 unpolarized) and the variational identity
    Tr[Sigma_J rho] = 2 eJ with Hermitian Sigma_J for a random complex rho."""
    ek = MF.ExchangeKernel(_jkernel(1.0, 0.3), SITEOF0, FLAVOROF0)
    assert ek.sf2idx.shape == (2, 2) and ek.sf2idx[0, 0] == 0 and ek.sf2idx[1, 1] == 3
    with pytest.raises(ValueError):
        MF.ExchangeKernel({(0, 0): np.array([[0.5, 0], [0, 0]], complex)}, SITEOF0, FLAVOROF0)
    with pytest.raises(ValueError):
        MF.ExchangeKernel(_jkernel(1.0, 0.0), [0, 0, 0, 0], FLAVOROF0)
    J1 = 0.7
    h = {(0, 0): np.zeros((4, 4), complex)}
    v = {(0, 0): np.zeros((4, 4), complex)}
    hf = MF.HartreeFock(h, v, exchange=MF.ExchangeKernel(_jkernel(J1, 0.0), SITEOF0, FLAVOROF0))
    hf({(0, 0): np.diag([1.0, 1.0, 0.0, 0.0]).astype(complex)})
    assert abs(hf.eJ + J1) < 1e-12
    hf({(0, 0): np.diag([0.5, 0.5, 0.5, 0.5]).astype(complex)})
    assert abs(hf.eJ + J1 / 2) < 1e-12
    rng = np.random.default_rng(7)
    r0 = rng.random((4, 4)) + 1j * rng.random((4, 4))
    r1 = rng.random((4, 4)) + 1j * rng.random((4, 4))
    rho = {(0, 0): (r0 + r0.conj().T) / 2, (1, 0): r1, (-1, 0): r1.conj().T}
    hf0 = MF.HartreeFock(h, v)(rho)
    hfJ = MF.HartreeFock(h, v, exchange=MF.ExchangeKernel(_jkernel(0.8, 0.35), SITEOF0, FLAVOROF0))(rho)
    SJ = {L: hfJ.hMF[L] - hf0.hMF.get(L, 0) for L in hfJ.hMF}
    for L in SJ:
        assert np.max(np.abs(SJ[L] - SJ[tuple(-x for x in L)].conj().T)) < 1e-12
    tr = sum(np.sum(rho[tuple(-x for x in L)].T * SJ[L]) for L in SJ if tuple(-x for x in L) in rho)
    assert abs(tr.real - 2 * hfJ.eJ) < 1e-10


def exchange_scf_case():
    """test/test_exchange.jl:85-123: two sites x two flavors, hopping t = 0.1 inside each
    flavor, U = 1 between different orbitals, J1 = 0.4."""
    t, U = 0.1, 1.0
    h1 = np.array([[0.0, t], [t, 0.0]], complex)
    h = {(0, 0): np.kron(np.eye(2), h1)}
    v = {(0, 0): (U * np.ones((4, 4)) - U * np.eye(4)).astype(complex)}
    return h, v


def test_exchange_scf_selects_polarized_state_oracle():
    """test/test_exchange.jl:85-123 on the oracle: with J the polarized solution wins by
    more than 0.3 J over the gain without J; every run converges and satisfies
    E = ekin + eH + eF + eJ."""
    h, v = exchange_scf_case()
    J1 = 0.4
    ks = L.regulargrid(8 * 8)
    Es = {}
    for label, occs, J in (("pol_J", [0.9, 0.9, 0.1, 0.1], J1), ("unp_J", [0.5] * 4, J1),
                           ("pol_0", [0.9, 0.9, 0.1, 0.1], None), ("unp_0", [0.5] * 4, None)):
        ek = MF.ExchangeKernel(_jkernel(J, 0.0), SITEOF0, FLAVOROF0) if J else None
        rho0 = {(0, 0): np.diag(occs).astype(complex)}
        rho, E, hf, conv, res, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, T=0.02, beta=0.5, tol=1e-9,
                                                        iterations=600, exchange=ek)
        assert conv
        assert abs(E - (hf.ekin + hf.eH + hf.eF + hf.eJ)) <= 1e-6 + 1e-8 * abs(E)
        Es[label] = E
    assert (Es["unp_J"] - Es["pol_J"]) - (Es["unp_0"] - Es["pol_0"]) > 0.3 * J1


def test_bdg_oracle_pins():
    """test/test_superconductivity.jl on the oracle: Nambu doubling gives +-E pairs,
    s-wave Delta = 0.25 opens +-Delta at the Dirac point, bond pairing stays Hermitian,
    the BdG kinetic energy of NN graphene at Gamma is -3, the filling with weak pairing
    at mu = 0 is 1/2, and the chemical potential reproduces its filling target."""
    from oracle import bdg as BDG
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    H = BDG.bdg_operator(h)
    for k in ([0.1, 0.2], [0.3, -0.1], [0.0, 0.0]):
        ev = np.sort(np.linalg.eigvalsh(K.fouriersum(H, k)))
        assert np.max(np.abs(ev + ev[::-1])) < 1e-10
    Hs = BDG.bdg_operator(h, {(0, 0): 0.25 * np.eye(2, dtype=complex)})
    ev = np.sort(np.linalg.eigvalsh(K.fouriersum(Hs, [1 / 3, -1 / 3])))
    assert abs(ev[2] - 0.25) < 1e-10 and abs(ev[1] + 0.25) < 1e-10
    bond = np.array([[0, 0.05], [0, 0]], complex)
    Hb = BDG.bdg_operator(h, {(1, 0): bond, (-1, 0): bond.conj().T})
    for k in ([0.1, 0.2], [1 / 3, -1 / 3]):
        Hk = K.fouriersum(Hb, k)
        assert np.max(np.abs(Hk - Hk.conj().T)) < 1e-12
        ev = np.sort(np.linalg.eigvalsh(Hk))
        assert np.max(np.abs(ev + ev[::-1])) < 1e-10
    z = (0, 0)
    _, e = BDG.bdg_densitymatrix(H, np.zeros((2, 1)), np.ones(1), 0.0, 1e-6, list(H.keys()))
    assert abs(e + 3.0) < 1e-3
    Hw = BDG.bdg_operator(h, {z: 0.05 * np.eye(2, dtype=complex)})
    assert abs(BDG.bdg_filling(Hw, L.regulargrid(12 * 12), 0.0, T=0.05) - 0.5) < 5e-3
    ks8 = L.regulargrid(8 * 8)
    Hp = BDG.bdg_operator(h, {z: 0.2 * np.eye(2, dtype=complex)})
    mu = BDG.bdg_chemicalpotential(Hp, ks8, 0.4, T=0.05)
    assert abs(BDG.bdg_filling(Hp, ks8, mu, T=0.05) - 0.4) < 1e-12


def test_bdg_pairing_functional_oracle_pins():
    """test/test_superconductivity.jl:230-275 on the oracle's HartreeFockBDG: the pairing
    field DeltaMF = v .* rhoD follows the phase of rhoD (phase covariance), and
    eP = 1/2 sum v |rhoD|^2 = -0.09 enters the double counting."""
    from oracle import bdg as BDG
    h = {(0,): np.zeros((2, 2), complex)}
    v = {(0,): np.array([[0, -1], [-1, 0]], complex)}
    F = np.array([[0, 1], [-1, 0]], complex)

    def pairing_update(theta):
        rho = BDG.bdg_operator({(0,): np.zeros((2, 2), complex)}, {(0,): np.exp(1j * theta) * F})
        hf = BDG.HartreeFockBDG(h, v, hartree=False, fock=True)(rho)
        return hf.DMF[(0,)].copy()

    th = 0.37 * math.pi
    D0, Dt = pairing_update(0.0), pairing_update(th)
    assert abs(Dt[0, 1] / D0[0, 1] - np.exp(1j * th)) < 1e-12
    assert abs(Dt[1, 0] / D0[1, 0] - np.exp(1j * th)) < 1e-12
    rho = BDG.bdg_operator({(0,): np.zeros((2, 2), complex)}, {(0,): np.array([[0, 0.3], [-0.3, 0]], complex)})
    hf = BDG.HartreeFockBDG(h, v, hartree=False, fock=True)(rho)
    assert abs(hf.eP + 0.09) < 1e-12
    assert abs(hf.doublecounting() - (hf.eH + hf.eF + hf.eP)) < 1e-14


def test_haldane_chern_pins():
    """test/test_haldane.jl:10-20,63-73,78-122 on the oracle: the Haldane model (t2 = 0.1,
    phi = +-pi/2) has E(K) = -+3 sqrt(3) t2, band Chern numbers +-1 on a 30 x 30 grid, and
    one gap at half filling with gap Chern number +-1."""
    for phi, sgn in ((math.pi / 2, 1), (-math.pi / 2, -1)):
        lat, h = M.haldane_model(t2=0.1, phi=phi)
        e = np.linalg.eigvalsh(K.fouriersum(h, [1 / 3, -1 / 3]))
        assert abs(e[0] + 0.5196152422706632) < 1e-12 and abs(e[1] - 0.5196152422706632) < 1e-12
        c = K.getcherns(h, 30, 30)
        assert abs(c[0] - sgn) < 0.05 and abs(c[1] + sgn) < 0.05
        gaps = K.gapcherns(h, 30, gaptol=1e-3)
        assert len(gaps) == 1 and gaps[0][0] == 1 and gaps[0][3] == sgn
        assert gaps[0][1] < 0 < gaps[0][2]


def test_fermisurface_density_known_answers():
    """Spectrum/fermisurface.jl on the oracle: a flat band at the requested energy gives
    1/pi at every k for any broadening; the :auto broadening is the mean band standard
    deviation over sqrt(nk); graphene's density on a 15 x 15 grid peaks near the Dirac
    points at E = 0."""
    ks = L.regulargrid(15 * 15)
    flat = {(0, 0): np.array([[0.3]], complex)}
    b, _ = K.bandmatrix(flat, ks)
    d, g = K.fermisurfacedensity_fromdata(b, [0.3], broadening=0.05)
    assert np.max(np.abs(d - 1 / math.pi)) < 1e-15 and g == 0.05
    h = M.nearestneighbor(L.honeycomb(), -1.0)
    b, _ = K.bandmatrix(h, ks)
    d, g = K.fermisurfacedensity_fromdata(b, [0.0, 1.0])
    assert abs(g - np.mean([np.std(x, ddof=1) for x in b]) / 15.0) < 1e-15
    assert np.argmax(d[0]) in [int(np.argmin(np.abs(b[0]))), int(np.argmin(np.abs(b[1])))]


def test_wilson_loop_winding_is_the_chern_number():
    """Wilson2D (Spectrum/berry.jl:258-327) on the oracle: the lower Haldane band's
    Wilson-loop phase winds once across the slices, +1 along one direction and -1 along
    the other for phi = pi/2, opposite for -pi/2 (its Chern number +-1)."""
    for phi, sgn in ((math.pi / 2, 1), (-math.pi / 2, -1)):
        _, h = M.haldane_model(t2=0.1, phi=phi)
        for direction, s_dir in ((1, 1), (2, -1)):
            en, _ = K.wilson_slices(h, 21, 21, [0], direction)
            d = (np.diff(np.append(en[:, 0], en[0, 0])) + 0.5) % 1.0 - 0.5
            assert abs(d.sum() - sgn * s_dir) < 1e-9


def test_chunked_k_reduction_matches_serial():
    """test/test_parallelism.jl:49-106: getdensitymatrix! on graphene (nearest
    neighbour, t = -1, 12^2 grid, mu = 0, T = 0.05) gives the same filling
    tr(rho_0)/2 and band energy whether the k-loop runs serially or as per-task
    partials folded at the end (atol 1e-10; the 8^2 case must not lose the energy
    scalar).  Here the partials are k-chunks with the global weights; half filling
    also follows from the particle-hole symmetry of the bipartite lattice."""
    h = M.nearestneighbor(L.honeycomb(), -1.0)
    for nk_lin in (12, 8):
        ks = L.regulargrid(nk_lin * nk_lin)
        nk = ks.shape[1]
        w = np.full(nk, 1.0 / nk)
        keys = list(h.keys())
        rho_s, eb_s = K.densitymatrix(h, ks, w, 0.0, 0.05, keys)
        rho_c = {R: np.zeros_like(rho_s[R]) for R in keys}
        eb_c = 0.0
        for chunk in np.array_split(np.arange(nk), 5):
            r, e = K.densitymatrix(h, ks[:, chunk], w[chunk], 0.0, 0.05, keys)
            for R in keys:
                rho_c[R] += r[R]
            eb_c += e
        f_s = np.real(np.trace(rho_s[(0, 0)])) / 2
        f_c = np.real(np.trace(rho_c[(0, 0)])) / 2
        assert abs(f_c - f_s) <= 1e-10 and abs(eb_c - eb_s) <= 1e-10
        assert abs(f_s - 0.5) <= 1e-12 and eb_s != 0.0


def test_hermitianize_pin():
    """test/test_tightbinding.jl:61-72: an onsite Hermitian block is Hermitian as Hops;
    a Hops whose R = +-1 blocks are not each other's adjoints is not, and
    hermitianize! repairs it (the SCF applies this to its initial guess,
    Meanfield/selfconsistent.jl:107-113,262-264)."""
    good = {(0, 0): np.array([[1, 1j], [-1j, 2]], complex)}
    assert MF.is_hermitian(good)
    bad = {(0, 0): np.array([[0, 1], [0, 0]], complex), (1, 0): np.array([[0, 0], [0, 1]], complex),
           (-1, 0): np.zeros((2, 2), complex)}
    assert not MF.is_hermitian(bad)
    MF.hermitianize(bad)
    assert MF.is_hermitian(bad)
    assert np.allclose(bad[(0, 0)], [[0, 0.5], [0.5, 0]]) and np.allclose(bad[(1, 0)], [[0, 0], [0, 0.5]])


def test_grid_and_path_shapes():
    """test/test_structure.jl:76-81,227-240: regulargrid returns the full requested
    grid (1000 points in 3D, 100 in 2D, first index fastest); kpath returns
    num_points 2D points; a sample that lands exactly on a tick is taken once."""
    assert L.regulargrid(1000, dim=3).shape == (3, 1000)
    g = L.regulargrid(100, dim=2)
    assert g.shape == (2, 100) and np.allclose(g[:, 1], [0.1, 0.0]) and np.allclose(g[:, 10], [0.0, 0.1])
    assert L.kpath(L.honeycomb(), 200).shape == (2, 200)

    class _Line:  # three collinear equidistant special points, unit reciprocal basis
        kdict = ({"a": (0.0, 0.0), "b": (1.0, 0.0), "c": (2.0, 0.0)}, ["a", "b", "c"])
        B = np.eye(2)

    p = L.kpath(_Line(), 5)
    assert p.shape == (2, 5) and np.allclose(p[0], [0.0, 0.5, 1.0, 1.5, 2.0]) and np.allclose(p[1], 0.0)


def test_interaction_range_beyond_hopping_range():
    """test/test_meanfield.jl:256-278: an interaction reaching farther than the
    hopping (onsite-only staggered h, gethubbard on 9 neighbour cells with a = 1.8,
    U = 2, mode sigma_x): the mean field gets blocks for keys(v) outside keys(h)
    (hartreefock.jl:191-205), its energies are finite, hMF is Hermitian as Hops, and
    the variational identity holds to 1e-10 on a 3 x 3 grid."""
    lat = L.honeycomb()
    h = {(0, 0): np.diag([0.3, 0.3, -0.3, -0.3]).astype(complex)}
    nbrs = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, -1), (1, -1), (-1, 1)]
    v = M.hubbard_v(lat, U=2.0, a=1.8, neighbors=nbrs)
    assert not set(v) <= set(h)
    rho = {R: np.zeros((4, 4), complex) for R in v}
    rho[(0, 0)] = M.antiferro_density(lat)
    hf = MF.HartreeFock(h, v)(rho)
    assert np.isfinite(hf.eH) and np.isfinite(hf.eF)
    assert set(hf.hMF) == set(h) | set(v) and MF.is_hermitian(hf.hMF)
    ks = np.array([[i / 3, j / 3] for j in range(3) for i in range(3)]).T

    def trprod(A, B):
        return sum(np.real(np.trace(K.fouriersum(A, k) @ K.fouriersum(B, k))) for k in ks.T) / ks.shape[1]

    assert abs(trprod(hf.hMF, rho) - trprod(h, rho) - 2 * (hf.eH + hf.eF)) < 1e-10


def test_hubbard_one_sided_neighbors_get_hermitian_partners():
    """gethops' hops! (Operators/gethops.jl:96-109) sets hops[-δL] = hops[δL]' for every
    nonzero δL and trim! drops all-zero blocks (TightBinding/types.jl:278-285): a
    one-sided neighbour list gives the same Hermitian V as the two-sided one."""
    lat = L.honeycomb()
    one = M.hubbard_v(lat, U=2.0, a=1.8, neighbors=[(0, 0), (1, 0)])
    two = M.hubbard_v(lat, U=2.0, a=1.8, neighbors=[(0, 0), (1, 0), (-1, 0)])
    assert set(one) == {(0, 0), (1, 0), (-1, 0)} == set(two)
    for R in one:
        assert np.array_equal(one[R], two[R])
        mR = tuple(-x for x in R)
        assert np.array_equal(one[mR], one[R].conj().T)
    far = M.hubbard_v(lat, U=2.0, a=0.5, neighbors=[(0, 0), (3, 0)])  # no pair within a = 0.5 at 3 cells
    assert set(far) == {(0, 0)}


def test_cpp_kloop_matches_python_oracle():
    """oracle/cpu_kspace.cpp (the C++/OpenMP restatement used as the timed CPU baseline and
    to generate the converged-SCF fixture) against the Python k-loop: bands, rho_L and the
    band energy, with and without weights, T > 0 and T = 0."""
    from oracle import cpu as C
    for name, h in M.batch_models()[:2] + [("c1", M.honeycomb_disorder()[1])]:
        ks = np.hstack([L.regulargrid(5 * 5), np.random.default_rng(3).random((2, 7))])
        nk = ks.shape[1]
        keys = list(h.keys())
        for w, T in ((np.full(nk, 1.0 / nk), 0.01), (np.random.default_rng(4).random(nk), 0.0)):
            r1, e1, b1 = C.densitymatrix(h, ks, w, 0.1, T, keys, want_bands=True)
            r2, e2 = K.densitymatrix(h, ks, w, 0.1, T, keys)
            assert max(np.max(np.abs(r1[R] - r2[R])) for R in keys) < 1e-12, name
            assert abs(e1 - e2) < 1e-12 * max(1.0, abs(e2)), name
            b2, _ = K.bandmatrix(h, ks)
            assert np.max(np.abs(b1 - b2)) < 1e-12 and np.max(np.abs(C.bandmatrix(h, ks) - b2)) < 1e-12, name
        r3, _ = C.densitymatrix(h, ks, None, 0.1, 0.01, keys)
        r4, _ = K.densitymatrix(h, ks, np.full(nk, 1.0 / nk), 0.1, 0.01, keys)
        assert max(np.max(np.abs(r3[R] - r4[R])) for R in keys) < 1e-12, name
