"""Parity of the batched blocked eigensolver (large-n path) with the oracle.

The blocked path is what orders beyond the one-CTA shared-memory plan run
(the twisted-bilayer workloads, n = 1324 and 2884).  Here it is also forced on
small orders (``set_blocked_min_n(1)``) so that every model and pin of the
plain path is checked through it.  Tolerances as in test_gpu_parity.py.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import kspace as K
from oracle import meanfield as MF
from lqm_workloads import lattice as L
from lqm_workloads import models as M

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
BAND_TOL = 1e-10
RHO_TOL = 1e-9


def rel_band_err(b, ref):
    return np.max(np.abs(b - ref)) / max(np.max(ref) - np.min(ref), 1.0)


@pytest.fixture(scope="module")
def bctx(lqm):
    c = lqm.Context(0, timeout=900)
    c.set_blocked_min_n(1)
    yield c
    c.close()


@pytest.fixture(scope="module")
def tbg10():
    return M.tbg_slater_koster(10)[1]


@pytest.fixture(scope="module")
def tsctx(lqm):
    """The blocked path with the two-stage reduction on every order it accepts (n > 17)."""
    c = lqm.Context(0, timeout=900)
    c.set_blocked_min_n(1)
    c.set_two_stage(1)
    yield c
    c.close()


def test_two_stage_models_bands_vectors_rho(lqm, tsctx):
    """Two-stage reduction (band of half-bandwidth 16, bulge chase, Q1 Q2 Z) on the
    batched workload's models and the n = 144 honeycomb: bands, eigenpairs and rho_L."""
    _, c1 = M.honeycomb_disorder()
    rng = np.random.default_rng(12)
    ks = np.hstack([L.regulargrid(6 * 6), rng.random((2, 7))])
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    for name, h in M.batch_models()[1:] + [("c1", c1)]:
        b, _ = lqm.bandmatrix(h, ks, ctx=tsctx)
        assert rel_band_err(b, K.bandmatrix(h, ks)[0]) <= BAND_TOL, name
        b2, U = lqm.bandmatrix(h, ks[:, :4], want_vectors=True, ctx=tsctx)
        n = b2.shape[0]
        for j in range(4):
            Hk = K.fouriersum(h, ks[:, j])
            assert np.max(np.abs(U[:, :, j].conj().T @ U[:, :, j] - np.eye(n))) < 1e-12, name
            assert np.max(np.abs(Hk @ U[:, :, j] - U[:, :, j] * b2[:, j])) < 1e-11, name
        keys = list(h.keys())
        rho = {R: None for R in keys}
        eb = lqm.getdensitymatrix(rho, h, ks, kweights=w, mu=0.0, T=0.01, ctx=tsctx)
        rref, ebref = K.densitymatrix(h, ks, w, 0.0, 0.01, keys)
        assert max(np.max(np.abs(rho[L_] - rref[L_])) for L_ in keys) <= RHO_TOL, name
        assert abs(eb - ebref) <= 1e-9 * max(1.0, abs(ebref)), name


def test_autotuner_picks_the_reduction_on_the_blocked_path(lqm):
    """On the blocked path (n = 256) the autotuner times the one- and the two-stage
    reduction for the sample's pass kind and keeps the faster; the tuned context's rho
    and eigenvectors still match the oracle."""
    c = lqm.Context(0, timeout=900)
    try:
        _, h = M.honeycomb_disorder(L_super=8)
        ks = L.regulargrid(16 * 16)
        for want_rho in (True, False):
            best, bms, table = lqm.autotune_eigh(h, ks, want_rho=want_rho, ctx=c)
            assert best in (0, 1) and sorted(table) == [0, 1] and bms == table[best] and bms > 0.0
        w = np.full(ks.shape[1], 1.0 / ks.shape[1])
        keys = list(h.keys())
        rho = {R: None for R in keys}
        lqm.getdensitymatrix(rho, h, ks, kweights=w, mu=0.0, T=0.01, ctx=c)
        rref, _ = K.densitymatrix(h, ks, w, 0.0, 0.01, keys)
        assert max(np.max(np.abs(rho[L_] - rref[L_])) for L_ in keys) <= RHO_TOL
        b, U = lqm.bandmatrix(h, ks[:, :3], want_vectors=True, ctx=c)
        for j in range(3):
            Hk = K.fouriersum(h, ks[:, j])
            assert np.max(np.abs(Hk @ U[:, :, j] - U[:, :, j] * b[:, j])) < 1e-11
        c.set_two_stage(1)
        with pytest.raises(lqm.LQMError):
            lqm.autotune_eigh(h, ks, ctx=c)
    finally:
        c.close()


def test_chase_bounded_wait_expiry_reports_and_recovers(lqm):
    """The bulge chase's inter-warp waits are bounded: with a limit of one poll the
    waits of the second and later sweeps run out at once (the sweep before them has not
    finished its first tasks), the kernel records the failure and stops, and the call
    returns LQM_EDEVICE; with the default limit the same context then gives the
    oracle's bands.  No fault is involved."""
    c = lqm.Context(0, timeout=600)
    try:
        _, h = M.honeycomb_disorder(L_super=8)  # n = 256: the blocked path, two-stage for bands
        ks = L.regulargrid(4 * 4)
        c.set_device_wait_limit(1)
        with pytest.raises(lqm.LQMError) as ei:
            lqm.bandmatrix(h, ks, ctx=c)
        assert ei.value.status == -6, ei.value
        c.set_device_wait_limit(0)
        b, _ = lqm.bandmatrix(h, ks, ctx=c)
        assert rel_band_err(b, K.bandmatrix(h, ks)[0]) <= BAND_TOL
    finally:
        c.close()


def test_two_stage_matches_one_stage(lqm, bctx, tsctx):
    """The same bands through both reductions of the blocked path, to rounding."""
    _, c1 = M.honeycomb_disorder()
    ks = np.random.default_rng(6).random((2, 200))
    one = lqm.Context(0, timeout=900)
    try:
        one.set_blocked_min_n(1)
        one.set_two_stage(0)
        for h in (M.batch_models()[2][1], c1):
            b1, _ = lqm.bandmatrix(h, ks, ctx=one)
            b2, _ = lqm.bandmatrix(h, ks, ctx=tsctx)
            assert rel_band_err(b2, b1) <= 1e-12
    finally:
        one.close()


def test_two_stage_hard_hermitian_inputs(lqm, tsctx):
    """The emulation suite's hard Hermitian inputs (n = 96) through the two-stage path."""
    from test_emulation import _hard_hermitian
    ks = np.zeros((2, 1))
    for name, Hk in _hard_hermitian():
        n = Hk.shape[0]
        if n <= 17:
            continue
        b, U = lqm.bandmatrix({(0, 0): Hk}, ks, want_vectors=True, ctx=tsctx)
        ref = K.eigh_upper(Hk, vectors=False)
        scale = max(np.max(np.abs(ref)), np.finfo(float).tiny)
        Uk = U[:, :, 0]
        assert np.all(np.isfinite(Uk)), name
        assert np.max(np.abs(b[:, 0] - ref)) <= 1e-12 * scale, name
        assert np.max(np.abs(Uk.conj().T @ Uk - np.eye(n))) <= 1e-12, name
        assert np.max(np.abs(Hk @ Uk - Uk * b[:, 0])) <= 1e-12 * scale, name


def test_blocked_tbg_golden_eigenvalues(lqm, bctx):
    pins = json.load(open(os.path.join(GOLD, "reference_pins.json")))["pins"]
    builders = {"honeycomb_twisted": L.honeycomb_twisted, "honeycomb_twisted_ABBA": L.honeycomb_twisted_ABBA,
                "honeycomb_twisted_ABAB": L.honeycomb_twisted_ABAB}
    from test_oracle_pins import pin_index
    for p in pins:
        h = M.graphene(builders[p["builder"]](p["N"]), tz=0.32)
        b, _ = lqm.bandmatrix(h, np.array(p["k"]).reshape(2, 1), ctx=bctx)
        i = pin_index(p["index"], b.shape[0])
        assert abs(b[i, 0] - p["value"]) <= p["atol"], p


def test_blocked_batch_models_bands_and_vectors(lqm, bctx):
    rng = np.random.default_rng(11)
    ks = np.hstack([L.regulargrid(8 * 8), rng.random((2, 9))])
    for name, h in M.batch_models():
        b, _ = lqm.bandmatrix(h, ks, ctx=bctx)
        assert rel_band_err(b, K.bandmatrix(h, ks)[0]) <= BAND_TOL, name
        b2, U = lqm.bandmatrix(h, ks[:, :5], want_vectors=True, ctx=bctx)
        n = b2.shape[0]
        for j in range(5):
            Hk = K.fouriersum(h, ks[:, j])
            assert np.max(np.abs(U[:, :, j].conj().T @ U[:, :, j] - np.eye(n))) < 1e-12, name
            assert np.max(np.abs(Hk @ U[:, :, j] - U[:, :, j] * b2[:, j])) < 1e-11, name


def test_blocked_densitymatrix_matches_oracle(lqm, bctx):
    _, c1 = M.honeycomb_disorder()
    for name, h in [("c1", c1)] + M.batch_models():
        ks = L.regulargrid(6 * 6)
        w = np.full(ks.shape[1], 1.0 / ks.shape[1])
        keys = list(h.keys())
        rho = {R: None for R in keys}
        eb = lqm.getdensitymatrix(rho, h, ks, mu=0.0, T=0.01, ctx=bctx)
        rref, ebref = K.densitymatrix(h, ks, w, 0.0, 0.01, keys)
        err = max(np.max(np.abs(rho[L_] - rref[L_])) for L_ in keys)
        assert err <= RHO_TOL, (name, err)
        assert abs(eb - ebref) <= 1e-9 * max(1.0, abs(ebref)), name


def test_blocked_matches_one_cta_path(lqm, ctx, bctx):
    """Same model through both eigensolvers: bands agree to rounding."""
    h = M.batch_models()[2][1]
    ks = np.random.default_rng(5).random((2, 300))
    b1, _ = lqm.bandmatrix(h, ks, ctx=ctx)
    b2, _ = lqm.bandmatrix(h, ks, ctx=bctx)
    assert rel_band_err(b2, b1) <= 1e-12


@pytest.mark.parametrize("two_stage", [1, 0])
def test_tbg_1324_bands_vectors_rho(lqm, ctx, tbg10, two_stage):
    """Twisted bilayer m=10 (n = 1324): beyond the one-CTA plan, so the default context
    takes the blocked path (both reductions).  Bands, eigenpairs and rho_L on a few k-points."""
    ctx.set_two_stage(two_stage)
    try:
        _tbg_1324_check(lqm, ctx, tbg10)
    finally:
        ctx.set_two_stage(-1)


def _tbg_1324_check(lqm, ctx, tbg10):
    h = tbg10
    n = next(iter(h.values())).shape[0]
    assert n == 1324
    ks = np.array([[0.0, 1 / 3, 0.137], [0.0, -1 / 3, 0.61]])
    b, U = lqm.bandmatrix(h, ks, want_vectors=True, ctx=ctx)
    ref = K.bandmatrix(h, ks)[0]
    assert rel_band_err(b, ref) <= BAND_TOL
    for j in range(ks.shape[1]):
        Hk = K.fouriersum(h, ks[:, j])
        assert np.max(np.abs(U[:, :, j].conj().T @ U[:, :, j] - np.eye(n))) < 1e-11
        assert np.max(np.abs(Hk @ U[:, :, j] - U[:, :, j] * b[:, j])) < 1e-10
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    keys = list(h.keys())
    rho = {R: None for R in keys}
    eb = lqm.getdensitymatrix(rho, h, ks, kweights=w, mu=0.0, T=0.01, ctx=ctx)
    rref, ebref = K.densitymatrix(h, ks, w, 0.0, 0.01, keys)
    assert max(np.max(np.abs(rho[L_] - rref[L_])) for L_ in keys) <= RHO_TOL
    assert abs(eb - ebref) <= 1e-9 * max(1.0, abs(ebref))


def test_tbg_1324_kpath_eigenvalues_only(lqm, ctx, tbg10):
    """Eigenvalue-only merges on the large path (the k-path part of the precision workload)."""
    h = tbg10
    ks = np.vstack([np.linspace(0, 0.5, 6), np.linspace(0, 0.25, 6)])
    b, _ = lqm.bandmatrix(h, ks, ctx=ctx)
    assert rel_band_err(b, K.bandmatrix(h, ks)[0]) <= BAND_TOL


def test_hubbard_scf_on_blocked_path_matches_oracle(lqm, bctx):
    """Hartree-Fock SCF at n = 128 (8x8 spinful triangular Hubbard): the eigen pass takes
    the blocked path, rho_k is formed by batched GEMMs, iterations 2+ replay a captured
    CUDA graph.  Same bounds as the n = 72 SCF test."""
    from oracle import meanfield as MF
    lat, h, v = M.triangular_hubbard(L_super=8)
    assert h[(0, 0)].shape[0] == 128
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=7)}
    ks = L.regulargrid(4 * 4)
    kw = dict(T=0.02, beta=0.3, tol=0.0, iterations=4)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=bctx, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, **kw)
    assert res.mf.iterations == it == 4
    assert np.max(np.abs(res.rho[(0, 0)] - rho_ref[(0, 0)])) <= RHO_TOL
    assert abs(res.energy - E_ref) <= 1e-9 * max(1.0, abs(E_ref))
    assert abs(res.mf.mu - hf_ref.mu) <= 1e-9
    assert abs(res.residual - resid) <= 1e-9


def test_screened_coulomb_hf_blocked_path_matches_oracle(lqm, bctx):
    """Hartree-Fock with the long-range screened Coulomb interaction on the twisted
    bilayer m=3 (n = 148, blocked path): Fock terms on every key of v, rho on the same
    keys.  Same bounds as the other SCF tests."""
    from oracle import meanfield as MF
    lat, h, v = M.tbg_screened_hf(3)
    n = h[(0, 0)].shape[0]
    assert n == 148
    rng = np.random.default_rng(11)
    X = rng.normal(size=(n, n)) * 0.01
    rho0 = {R: np.zeros((n, n), complex) for R in v}
    rho0[(0, 0)] = 0.5 * np.eye(n) + (X + X.T)
    ks = L.regulargrid(4 * 4)
    kw = dict(T=0.05, beta=0.3, tol=0.0, iterations=4)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=bctx, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, **kw)
    assert res.mf.iterations == it == 4
    assert max(np.max(np.abs(res.rho[R] - rho_ref[R])) for R in rho0) <= RHO_TOL
    assert abs(res.energy - E_ref) <= 1e-9 * max(1.0, abs(E_ref))
    assert abs(res.mf.mu - hf_ref.mu) <= 1e-9


@pytest.mark.parametrize("blocked", [False, True], ids=["default", "blocked"])
def test_band_expectation_values_match_oracle(lqm, ctx, bctx, blocked):
    """bandmatrix(H, ks, projectors...) through lqm_bandmatrix_obs: a k-independent
    random Hermitian matrix, H itself (k-dependent Hops: obs = bands) and the identity."""
    c = bctx if blocked else ctx
    rng = np.random.default_rng(13)
    cases = M.batch_models() + [("honeycomb144", M.honeycomb_disorder()[1])]
    for name, h in cases:
        n = h[(0, 0)].shape[0]
        X = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        P = X + X.conj().T
        ks = rng.random((2, 7))
        res = lqm.getbands(h, ks, [P, h, np.eye(n)], ctx=c)
        bref, oref = K.bandmatrix_obs(h, ks, [P, h, np.eye(n)])
        scale = max(np.max(bref) - np.min(bref), 1.0)
        assert np.max(np.abs(res.bands - bref)) <= BAND_TOL * scale, name
        # within a degenerate group (spin pairs) only the sum of <u|P|u> is basis-independent
        for j in range(ks.shape[1]):
            b_ = bref[:, j]
            start = 0
            for i in range(1, n + 1):
                if i == n or b_[i] - b_[i - 1] > 1e-8 * scale:
                    g = slice(start, i)
                    d = abs(res.obs[g, j, 0].sum() - oref[g, j, 0].sum())
                    assert d <= 1e-10 * np.max(np.abs(P)) * n, (name, j, start, i)
                    start = i
        assert np.max(np.abs(res.obs[:, :, 1] - res.bands)) <= BAND_TOL * scale, name
        assert np.max(np.abs(res.obs[:, :, 2] - 1.0)) <= 1e-12, name


@pytest.mark.parametrize("blocked", [False, True], ids=["default", "blocked"])
def test_density_and_ldos_match_oracle(lqm, ctx, bctx, blocked):
    """density (dos.jl:20-52) and ldos (dos.jl:56-98) through lqm_density / lqm_ldos:
    basis-independent per-orbital sums, so degenerate bands do not matter."""
    c = bctx if blocked else ctx
    cases = M.batch_models() + [("honeycomb144", M.honeycomb_disorder()[1])]
    ks = L.regulargrid(6 * 6)
    for name, h in cases:
        n_ref = K.density(h, ks, mu=0.1)
        assert np.max(np.abs(lqm.density(h, ks, mu=0.1, ctx=c) - n_ref)) <= 1e-12 * h[(0, 0)].shape[0], name
        for om in ([0.2], [-1.0, 0.0, 0.7]):
            ld_ref = K.ldos(h, ks, om, gamma=0.05)
            ld = lqm.ldos(h, ks, om, gamma=0.05, ctx=c)
            assert np.max(np.abs(ld - ld_ref)) <= 1e-10 * max(1.0, np.max(ld_ref)), (name, om)


def test_berry_plaquettes_match_oracle(lqm, ctx):
    """berry(H, NX, NY, bandindices) through lqm_berry against the oracle: gapped graphene
    (one band) and the spin-orbit triangular model (its four lowest bands, whole
    degenerate groups so the plaquette phases are gauge invariant)."""
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    h[(0, 0)] = h[(0, 0)] + np.diag([0.3, -0.3])
    _, F = lqm.berry(h, 12, 12, [0], ctx=ctx)
    assert np.max(np.abs(F - K.berry(h, 12, 12, [0]))) <= 1e-10
    h3 = M.batch_models()[2][1]
    _, F3 = lqm.berry(h3, 8, 8, [0, 1, 2, 3], ctx=ctx)
    assert np.max(np.abs(F3 - K.berry(h3, 8, 8, [0, 1, 2, 3]))) <= 1e-10
    assert abs(F3.sum()) <= 1e-9  # integer total (zero for this model)


def test_optical_conductivity_matches_oracle(lqm, ctx, bctx):
    """opticalconductivity(frequencies, H, J1, J2, ks; mu, Gamma, T) through
    lqm_opticalconductivity against the oracle: graphene on the klin=30 grid of
    test/test_linearresponse.jl (with its sigma invariants on the device result), and
    the disordered spinful honeycomb 6x6 cell (n=144) on both eigensolver paths."""
    lat = L.honeycomb()
    h = M.graphene(lat)
    Js = M.currentoperators(lat, h)
    om = np.linspace(0.05, 3.0, 30)
    gam, T, mu = 0.05, 0.01, 0.0
    ks = L.regulargrid(nk=30 ** 2)
    sig = {}
    for a, b in ((0, 0), (1, 1), (0, 1)):
        chi = lqm.opticalconductivity(om, h, Js[a], Js[b], ks, mu=mu, Gamma=gam, T=T, ctx=ctx)
        ref = K.opticalconductivity(om, h, Js[a], Js[b], ks, mu, gam, T)
        assert np.max(np.abs(chi - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref))), (a, b)
        sig[a, b] = -(chi - chi[0]) / (om + 1j * gam)
    assert np.max(np.abs(sig[0, 0].real - sig[1, 1].real)) < 1e-10
    assert np.max(np.abs(sig[0, 1].real)) < 1e-10
    assert np.all(sig[0, 0].real > -1e-6)

    lat6, h6 = M.honeycomb_disorder(6)
    J6 = M.currentoperators(lat6, h6)
    rng = np.random.default_rng(11)
    ks6 = rng.uniform(-0.5, 0.5, (2, 6))
    om6 = np.linspace(0.0, 4.0, 21)
    ref = K.opticalconductivity(om6, h6, J6[0], J6[1], ks6, 0.05, 0.04, 0.1)
    c1 = lqm.Context(0, timeout=900)
    c1.set_blocked_min_n(10 ** 9)  # the one-CTA eigensolver
    try:
        for c in (c1, bctx):
            chi = lqm.opticalconductivity(om6, h6, J6[0], J6[1], ks6, mu=0.05, Gamma=0.04, T=0.1, ctx=c)
            assert np.max(np.abs(chi - ref)) <= 1e-9 * max(1.0, np.max(np.abs(ref)))
    finally:
        c1.close()


def test_partial_spectrum_matches_oracle(lqm, ctx):
    """bandmatrix / getdensitymatrix! with format=:sparse, num_bands through
    lqm_bandmatrix_partial and lqm_densitymatrix_partial: the selection tests of
    test/test_eigen.jl:11-85 (a seeded 60 x 60 matrix as a single-key Hops: :LM at
    sigma = 0 and 0.2, :SR, :LR, ascending, residuals, determinism), the residual and
    orthonormality contract of test/test_eigen.jl:42-65 on the twisted bilayer N = 5
    (n = 364, blocked eigensolver) against the oracle, and the partial density matrix
    on the disordered honeycomb 6x6 cell."""
    rng = np.random.default_rng(0x123456789ABCDEF)
    A = rng.random((60, 60)) - 0.5
    A = np.triu(A) + np.triu(A, 1).T
    h = {(0, 0): A.astype(complex)}
    ks = np.zeros((2, 1))
    e = np.sort(np.linalg.eigvalsh(A))
    lm, _ = lqm.bandmatrix_partial(h, ks, 10, sigma=0.0, ctx=ctx)
    assert np.allclose(lm[:, 0], np.sort(sorted(e, key=abs)[:10]), atol=1e-10)
    sr, _ = lqm.bandmatrix_partial(h, ks, 10, which="SR", ctx=ctx)
    lr, _ = lqm.bandmatrix_partial(h, ks, 10, which=":LR", ctx=ctx)
    assert np.allclose(sr[:, 0], e[:10], atol=1e-10) and np.allclose(lr[:, 0], e[-10:], atol=1e-10)
    for which, sig in (("LM", 0.2), ("SR", 1e-8), ("LR", 1e-8)):
        b, U = lqm.bandmatrix_partial(h, ks, 6, sigma=sig, which=which, want_vectors=True, ctx=ctx)
        assert np.all(np.diff(b[:, 0]) >= 0)
        assert np.max(np.abs(A @ U[:, :, 0] - U[:, :, 0] * b[:, 0][None, :])) < 1e-8
        ref, _ = K.bandmatrix_partial(h, ks, 6, sigma=sig, which=which)
        assert np.max(np.abs(b - ref)) < 1e-10
    b1, _ = lqm.bandmatrix_partial(h, ks, 4, ctx=ctx)
    b2, _ = lqm.bandmatrix_partial(h, ks, 4, ctx=ctx)
    assert np.array_equal(b1, b2)

    lat = L.honeycomb_twisted(5)
    ht = M.graphene(lat)
    kp = L.kpath(lat, 4)[:, 1:3]
    b, U = lqm.bandmatrix(ht, kp, format="sparse", num_bands=10, want_vectors=True, ctx=ctx)
    ref, _ = K.bandmatrix_partial(ht, kp, 10)
    assert rel_band_err(b, ref) <= BAND_TOL
    for j in range(kp.shape[1]):
        Hk = K.fouriersum(ht, kp[:, j])
        Uj = U[:, :, j]
        assert max(np.linalg.norm(Hk @ Uj[:, m] - b[m, j] * Uj[:, m]) for m in range(10)) < 1e-9
        assert np.linalg.norm(Uj.conj().T @ Uj - np.eye(10), 2) < 1e-10

    _, h6 = M.honeycomb_disorder(6)
    ks6 = rng.uniform(-0.5, 0.5, (2, 16))
    w6 = np.full(16, 1.0 / 16)
    rho = {R: None for R in M.KEYS9}
    eb = lqm.getdensitymatrix(rho, h6, ks6, mu=0.0, T=0.01, format="sparse", num_bands=24, ctx=ctx)
    rref, ebref = K.densitymatrix_partial(h6, ks6, w6, 0.0, 0.01, M.KEYS9, 24)
    assert max(np.max(np.abs(rho[R] - rref[R])) for R in M.KEYS9) <= RHO_TOL
    assert abs(eb - ebref) <= 1e-10 * max(1.0, abs(ebref))


def test_exchange_scf_blocked_path_matches_oracle(lqm, ctx):
    """J-augmented SCF on the blocked eigensolver path: the disordered spinful honeycomb
    6x6 cell (n = 144, 72 sites x 2 spin flavors, spin the fast index) with Hubbard U = 2
    and a nearest-neighbour exchange kernel J = 0.1 on every bond (its zero-key diagonal
    empty), 4 iterations from a random local magnetization, against the oracle."""
    lat, h = M.honeycomb_disorder(6)
    v = M.hubbard_v(lat, U=2.0)
    nn_site = M.nearestneighbor(lat, -1.0)
    j = {R: 0.1 * (np.abs(B) > 0).astype(complex) for R, B in nn_site.items()}
    ns = lat.norb
    siteof = [I // 2 for I in range(2 * ns)]
    flavorof = [I % 2 for I in range(2 * ns)]
    rho0 = {R: np.zeros((2 * ns, 2 * ns), complex) for R in M.KEYS9}
    rho0[(0, 0)] = M.random_local_magnetization(ns, seed=4)
    ks = L.regulargrid(4 * 4)
    kw = dict(T=0.05, beta=0.4, tol=0.0, iterations=4)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, exchange=lqm.ExchangeKernel(j, siteof, flavorof), **kw)
    rho_ref, E_ref, hf_ref, _, _, it = MF.solvehartreefock(h, v, rho0, 0.5, ks,
                                                           exchange=MF.ExchangeKernel(j, siteof, flavorof), **kw)
    assert res.mf.iterations == it == 4
    assert max(np.max(np.abs(res.rho[R] - rho_ref[R])) for R in M.KEYS9) <= RHO_TOL
    assert abs(res.energy - E_ref) <= 1e-9 * max(1.0, abs(E_ref))
    assert abs(res.mf.eJ - hf_ref.eJ) <= 1e-9 * max(1.0, abs(hf_ref.eJ))


def test_chern_numbers_match_oracle(lqm, ctx):
    """getcherns / spectralgaps / gapcherns (Spectrum/berry.jl:378-487) through
    lqm_berry_flux and the device bands: the Haldane cases of test/test_haldane.jl:78-122
    (band Chern numbers +-1, one gap at half filling with Chern +-1), and parity of the
    unrounded band fluxes with the oracle on the spin-orbit triangular model (n = 96)."""
    for phi, sgn in ((math.pi / 2, 1), (-math.pi / 2, -1)):
        _, h = M.haldane_model(t2=0.1, phi=phi)
        c = lqm.getcherns(h, 30, 30, ctx=ctx)
        assert abs(c[0] - sgn) < 0.05 and abs(c[1] + sgn) < 0.05
        assert max(abs(a - b) for a, b in zip(c, K.getcherns(h, 30, 30))) <= 1e-10
        gaps = lqm.gapcherns(h, 30, gaptol=1e-3, ctx=ctx)
        assert len(gaps) == 1 and gaps[0][0] == 1 and gaps[0][3] == sgn and gaps[0][1] < 0 < gaps[0][2]
        ref = K.gapcherns(h, 30, gaptol=1e-3)
        assert abs(gaps[0][1] - ref[0][1]) <= 1e-12 and abs(gaps[0][2] - ref[0][2]) <= 1e-12
    h3 = M.batch_models()[2][1]
    sets = [[0, 1, 2, 3], [0, 1], list(range(8))]
    flux = lqm.berry_flux(h3, 8, 8, sets, ctx=ctx)
    for f, s_ in zip(flux, sets):
        assert abs(f - float(np.sum(K.berry(h3, 8, 8, s_)))) <= 1e-9


def test_berry_along_path_matches_oracle(lqm, ctx):
    """berryalongpath(H, kpoints) (Spectrum/berry.jl:170-238) through lqm_berry_path against
    the oracle: the Haldane model (gapped, non-degenerate bands) along its 60-point
    Gamma-K-M-K'-Gamma-M path, and the two bands' phases of opposite sign at each point."""
    lat, h = M.haldane_model(t2=0.1, phi=math.pi / 2)
    kp = L.kpath(lat, 60)
    b = lqm.berryalongpath(h, kp, ctx=ctx)
    ref = K.berryalongpath(h, kp)
    assert b.shape == ref.shape
    assert np.max(np.abs(b - ref)) <= 1e-9
    assert np.max(np.abs(b[0] + b[1])) <= 1e-9  # the two bands' curvatures cancel


def test_fermisurface_density_matches_oracle(lqm, ctx):
    """fermisurfacedensity (Spectrum/fermisurface.jl) through lqm_fermisurface against the
    oracle: graphene on the default 15 x 15 grid with the :auto broadening, the disordered
    honeycomb 6x6 cell (n = 144, blocked eigensolver) with a fixed broadening, and the
    weighted form with the sublattice-0 projector's band expectation values."""
    h = M.nearestneighbor(L.honeycomb(), -1.0)
    ks, d, g = lqm.fermisurfacedensity(h, [0.0, 0.5, 1.0], ctx=ctx)
    b, _ = K.bandmatrix(h, ks)
    ref, gref = K.fermisurfacedensity_fromdata(b, [0.0, 0.5, 1.0])
    assert abs(g - gref) <= 1e-14 and np.max(np.abs(d - ref)) <= 1e-9 * np.max(ref)
    lat6, h6 = M.honeycomb_disorder(6)
    rng = np.random.default_rng(3)
    ks6 = rng.uniform(-0.5, 0.5, (2, 40))
    E = np.linspace(-1.0, 1.0, 9)
    _, d6, g6 = lqm.fermisurfacedensity(h6, E, ks=ks6, broadening=0.05, ctx=ctx)
    b6, _ = K.bandmatrix(h6, ks6)
    ref6, _ = K.fermisurfacedensity_fromdata(b6, E, broadening=0.05)
    assert g6 == 0.05 and np.max(np.abs(d6 - ref6)) <= 1e-9 * np.max(ref6)
    P = np.diag(np.repeat((lat6.extracoord("sublattice") == 0).astype(float), 2)).astype(complex)
    bo, obs = lqm.bandmatrix_obs(h6, ks6, [P], ctx=ctx)
    _, dw, _ = lqm.fermisurfacedensity(h6, E, ks=ks6, broadening=0.05, obs=obs[:, :, 0], ctx=ctx)
    refw, _ = K.fermisurfacedensity_fromdata(b6, E, obs=obs[:, :, 0], broadening=0.05)
    assert np.max(np.abs(dw - refw)) <= 1e-9 * np.max(np.abs(refw))


def test_wilson_loops_match_oracle(lqm, ctx):
    """Wilson loops (WilsonSlice1D / Wilson2D, Spectrum/berry.jl:258-367) through lqm_wilson
    against the oracle: the lower Haldane band (one band; its phase winds by the Chern
    number) in both directions, and the four lowest bands of the spin-orbit triangular model
    (whole degenerate pairs), whose eigenvectors also diagonalise the loop the oracle builds."""
    _, h = M.haldane_model(t2=0.1, phi=math.pi / 2)
    for direction, wind in ((1, 1), (2, -1)):
        en, _ = lqm.wilson_slices(h, 21, 21, [0], direction, ctx=ctx)
        ref, _ = K.wilson_slices(h, 21, 21, [0], direction)
        assert np.max(np.abs(en - ref)) <= 1e-9
        d = (np.diff(np.append(en[:, 0], en[0, 0])) + 0.5) % 1.0 - 0.5
        assert abs(d.sum() - wind) < 1e-9
    h3 = M.batch_models()[2][1]
    en1, U1, en2, U2 = lqm.wilson2d(h3, 9, 9, [0, 1, 2, 3], ctx=ctx)
    for en, U, direction in ((en1, U1, 1), (en2, U2, 2)):
        ref, _ = K.wilson_slices(h3, 9, 9, [0, 1, 2, 3], direction)
        assert np.max(np.abs(en - ref)) <= 1e-9
        for u in U:
            assert np.max(np.abs(u.conj().T @ u - np.eye(4))) <= 1e-12


def test_wilson_wannier_matches_oracle(lqm, ctx):
    """WilsonWannier2D (Spectrum/berry.jl:274-301) through lqm_wilson_wannier against the
    oracle: the lower band of the Haldane model and of gapped graphene on a 13 x 13 grid.
    (The rotation is gauge invariant only for non-degenerate loop spectra: a band set
    spanning every band, for one, has the identity as its loop and no preferred
    eigenvectors.)"""
    _, h = M.haldane_model(t2=0.1, phi=math.pi / 2)
    h0 = M.nearestneighbor(L.honeycomb(), -1.0)
    h0[(0, 0)] = h0[(0, 0)] + np.diag([0.3, -0.3])
    for hh, bands in ((h, [0]), (h0, [0])):
        p1, p2 = lqm.wilson_wannier2d(hh, 13, 13, bands, ctx=ctx)
        r1, r2 = K.wilson_wannier2d(hh, 13, 13, bands)
        assert np.max(np.abs(p1 - np.array(r1))) <= 1e-9 and np.max(np.abs(p2 - np.array(r2))) <= 1e-9
