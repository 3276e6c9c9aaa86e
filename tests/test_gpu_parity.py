"""Parity of the CUDA path (through the C-ABI) with the CPU oracle and the reference's pins.

Tolerances (FP64 plain path): bands within 1e-10 of the spectral width, rho_L and
converged mean fields within 1e-9 (absolute, entries are O(1)), mu within 1e-12.
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

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
BAND_TOL = 1e-10
RHO_TOL = 1e-9


def rel_band_err(b, ref):
    return np.max(np.abs(b - ref)) / max(np.max(ref) - np.min(ref), 1.0)


def oracle_bands(h, ks):
    return K.bandmatrix(h, ks)[0]


@pytest.fixture(scope="module")
def c1():
    _, h = M.honeycomb_disorder()
    return h


# ---------------------------------------------------------------- golden pins
def test_tbg_golden_eigenvalues(lqm, ctx):
    pins = json.load(open(os.path.join(GOLD, "reference_pins.json")))["pins"]
    builders = {"honeycomb_twisted": L.honeycomb_twisted, "honeycomb_twisted_ABBA": L.honeycomb_twisted_ABBA,
                "honeycomb_twisted_ABAB": L.honeycomb_twisted_ABAB}
    from test_oracle_pins import pin_index
    for p in pins:
        h = M.graphene(builders[p["builder"]](p["N"]), tz=0.32)
        b, _ = lqm.bandmatrix(h, np.array(p["k"]).reshape(2, 1), ctx=ctx)
        i = pin_index(p["index"], b.shape[0])
        assert abs(b[i, 0] - p["value"]) <= p["atol"], p


def test_graphene_analytic_bands(lqm, ctx):
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    ks = L.kpath(lat, 200)
    b = lqm.getbands(h, ks, ctx=ctx).bands
    from test_oracle_pins import graphene_conduction
    up = np.array([graphene_conduction(k) for k in ks.T])
    assert np.sum(np.abs(b[0] + up)) + np.sum(np.abs(b[1] - up)) < 1e-12


def test_square_analytic_bands(lqm, ctx):
    lat = L.square()
    h = M.nearestneighbor(lat, -1.0)
    ks = L.kpath(lat, 200)
    b, _ = lqm.bandmatrix(h, ks, ctx=ctx)
    ana = -2 * (np.cos(2 * np.pi * ks[0]) + np.cos(2 * np.pi * ks[1]))
    assert np.max(np.abs(b[0] - ana)) < 1e-12


# ---------------------------------------------------------------- bands
def test_c1_bands_full_grid(lqm, ctx, c1):
    ks = L.regulargrid(48 * 48)
    b, _ = lqm.bandmatrix(c1, ks, ctx=ctx)
    sub = np.arange(0, ks.shape[1], 7)
    ref = oracle_bands(c1, ks[:, sub])
    assert rel_band_err(b[:, sub], ref) <= BAND_TOL


def test_batch_models_bands(lqm, ctx):
    rng = np.random.default_rng(7)
    ks = np.hstack([L.regulargrid(16 * 16), rng.random((2, 40))])
    for name, h in M.batch_models():
        b, _ = lqm.bandmatrix(h, ks, ctx=ctx)
        assert rel_band_err(b, oracle_bands(h, ks)) <= BAND_TOL, name


def test_hops_upload_free_reuse(lqm):
    """Upload, one pass and free in a loop, the way a per-call user does: the context
    hands freed Hops buffers to later uploads (of other orders and key counts too, so
    the keys sit at another offset of a reused buffer), and every pass still matches
    the oracle."""
    c = lqm.Context(0, timeout=600)
    try:
        ks = np.hstack([L.regulargrid(8 * 8), np.random.default_rng(3).random((2, 16))])
        models = [h for _, h in M.batch_models()]
        models.append({R: models[0][R] for R in [(0, 0), (1, 0), (-1, 0)]})  # fewer keys, same order
        ref = [oracle_bands(h, ks) for h in models]
        for it in range(3):
            for h, r in zip(models if it % 2 == 0 else models[::-1], ref if it % 2 == 0 else ref[::-1]):
                Hd = lqm.DeviceHops(h, c)
                b, _ = lqm.bandmatrix(Hd, ks, ctx=c)
                Hd.free()
                assert rel_band_err(b, r) <= BAND_TOL
    finally:
        c.close()


def test_stats_modes(lqm):
    """reset_stats(timing=True) times the eigensolver launches without its phase
    counters; reset_stats(phases=True) records both."""
    c = lqm.Context(0, timeout=600)
    try:
        h = M.batch_models()[1][1]
        ks = L.regulargrid(8 * 8)
        c.reset_stats(timing=True)
        lqm.bandmatrix(h, ks, ctx=c)
        ms, launches, _ = c.stats()
        assert launches >= 1 and ms > 0.0
        assert all(v == 0.0 for v in c.phase_cycles())
        c.reset_stats(phases=True)
        lqm.bandmatrix(h, ks, ctx=c)
        ph = c.phase_cycles()
        assert c.stats()[1] >= 1 and ph[1] > 0.0 and ph[2] > 0.0
        c.reset_stats(timing=False)
    finally:
        c.close()


def test_large_n_global_scratch_path(lqm):
    # n = 148 on the one-CTA kernel (forced, whatever the default switch): the
    # Householder matrix lives in global scratch (does not fit shared memory)
    ctx = lqm.Context(0, timeout=600)
    ctx.set_blocked_min_n(10 ** 9)
    h = M.graphene(L.honeycomb_twisted(3), tz=0.32)
    ks = np.array([[0.0, 1 / 3, 0.21], [0.0, -1 / 3, 0.55]])
    b, U = lqm.bandmatrix(h, ks, want_vectors=True, ctx=ctx)
    assert rel_band_err(b, oracle_bands(h, ks)) <= BAND_TOL
    for j in range(ks.shape[1]):
        Hk = K.fouriersum(h, ks[:, j])
        assert np.max(np.abs(U[:, :, j].conj().T @ U[:, :, j] - np.eye(148))) < 1e-12
        assert np.max(np.abs(Hk @ U[:, :, j] - U[:, :, j] * b[:, j])) < 1e-11


def test_eigenvectors_orthonormal_residual(lqm, ctx, c1):
    ks = L.regulargrid(6 * 6)
    b, U = lqm.bandmatrix(c1, ks, want_vectors=True, ctx=ctx)
    n = b.shape[0]
    for j in range(ks.shape[1]):
        Hk = K.fouriersum(c1, ks[:, j])
        Uj = U[:, :, j]
        assert np.max(np.abs(Uj.conj().T @ Uj - np.eye(n))) < 1e-12
        assert np.max(np.abs(Hk @ Uj - Uj * b[:, j])) < 1e-11


def test_edge_cases_small_n_and_single_k(lqm, ctx):
    h1 = {(0, 0): np.array([[0.25]], complex), (1, 0): np.array([[-0.5]], complex),
          (-1, 0): np.array([[-0.5]], complex)}
    ks = np.array([[0.1, 0.5], [0.0, 0.0]])
    b, U = lqm.bandmatrix(h1, ks, want_vectors=True, ctx=ctx)
    assert np.allclose(b[0], 0.25 - np.cos(2 * np.pi * ks[0]), atol=1e-14)
    assert np.allclose(np.abs(U[0, 0, :]), 1.0)
    h = M.batch_models()[0][1]
    b, _ = lqm.bandmatrix(h, np.array([[0.3], [0.1]]), ctx=ctx)
    assert rel_band_err(b, oracle_bands(h, np.array([[0.3], [0.1]]))) <= BAND_TOL


def test_bloch_sum(lqm, ctx, c1):
    ks = np.array([[0.0, 0.25, 0.7], [0.0, 0.5, 0.11]])
    Hk = lqm.bloch(c1, ks, ctx=ctx)
    for j in range(3):
        assert np.max(np.abs(Hk[:, :, j] - K.fouriersum(c1, ks[:, j]))) < 1e-13


def test_deterministic(lqm, ctx, c1):
    ks = L.regulargrid(8 * 8)
    b1, _ = lqm.bandmatrix(c1, ks, ctx=ctx)
    b2, _ = lqm.bandmatrix(c1, ks, ctx=ctx)
    assert np.array_equal(b1, b2)
    r1, r2 = {R: None for R in c1}, {R: None for R in c1}
    e1 = lqm.getdensitymatrix(r1, c1, ks, mu=0.0, T=0.01, ctx=ctx)
    e2 = lqm.getdensitymatrix(r2, c1, ks, mu=0.0, T=0.01, ctx=ctx)
    assert e1 == e2 and all(np.array_equal(r1[R], r2[R]) for R in r1)


# ---------------------------------------------------------------- density matrix
def test_c1_densitymatrix(lqm, ctx, c1):
    ks = L.regulargrid(12 * 12)
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    rho = {R: None for R in c1}
    eb = lqm.getdensitymatrix(rho, c1, ks, mu=0.0, T=0.01, ctx=ctx)
    ref, eb_ref = K.densitymatrix(c1, ks, w, 0.0, 0.01, list(c1.keys()))
    for R in c1:
        assert np.max(np.abs(rho[R] - ref[R])) <= RHO_TOL, R
    assert abs(eb - eb_ref) <= 1e-9 * max(1.0, abs(eb_ref))


def test_densitymatrix_weights_and_zero_T(lqm, ctx):
    h = M.graphene(L.honeycomb(), spin=True)
    nk = 9
    ks = np.array([[i / nk, j / nk] for j in range(nk) for i in range(nk)]).T
    rng = np.random.default_rng(3)
    w = rng.random(ks.shape[1])
    w /= w.sum()
    rho = {R: None for R in h}
    eb = lqm.getdensitymatrix(rho, h, ks, kweights=w, mu=-0.5, T=0.0, ctx=ctx)
    ref, eb_ref = K.densitymatrix(h, ks, w, -0.5, 0.0, list(h.keys()))
    for R in h:
        assert np.max(np.abs(rho[R] - ref[R])) <= RHO_TOL
    assert abs(eb - eb_ref) < 1e-10


def test_batch_models_densitymatrix(lqm, ctx):
    ks = L.regulargrid(8 * 8)
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    for name, h in M.batch_models():
        rho = {R: None for R in h}
        eb = lqm.getdensitymatrix(rho, h, ks, mu=0.0, T=0.01, ctx=ctx)
        ref, eb_ref = K.densitymatrix(h, ks, w, 0.0, 0.01, list(h.keys()))
        for R in h:
            assert np.max(np.abs(rho[R] - ref[R])) <= RHO_TOL, (name, R)
        assert abs(eb - eb_ref) <= 1e-9 * max(1.0, abs(eb_ref))


# ---------------------------------------------------------------- mu, DOS
@pytest.mark.parametrize("T,filling", [(0.01, 0.5), (0.05, 0.3), (0.0, 0.5), (0.0, 0.37), (0.0, 1.0), (0.0, 0.0)])
def test_chemicalpotential(lqm, ctx, c1, T, filling):
    ks = L.regulargrid(8 * 8)
    mu = lqm.chemicalpotential(c1, ks, filling, T=T, ctx=ctx)
    ref = K.chemicalpotential(oracle_bands(c1, ks), filling, T)
    assert abs(mu - ref) <= 1e-12 * max(1.0, abs(ref))


def test_dos(lqm, ctx):
    for name, h in M.batch_models()[:2]:
        ks = L.regulargrid(16 * 16)
        b = oracle_bands(h, ks)
        om = np.linspace(b.min(), b.max(), 500)
        dos = lqm.getdos(h, om, ks, 0.05, ctx=ctx)
        ref = K.dos_from_bands(b, om, 0.05)
        assert np.max(np.abs(dos - ref)) <= 1e-10 * np.max(ref), name


def test_graphene_dos_invariants(lqm, ctx):
    h = M.nearestneighbor(L.honeycomb(), -1.0)
    om = np.linspace(-3.05, 3.05, 401)
    dos = lqm.getdos(h, om, L.regulargrid(120 * 120), 0.05, ctx=ctx)
    assert np.max(np.abs(dos - dos[::-1])) / np.max(np.abs(dos)) < 1e-10
    assert abs(np.sum(dos) * (om[1] - om[0]) - 2 * math.pi) / (2 * math.pi) < 0.05


# ---------------------------------------------------------------- SCF
def test_hubbard_scf_matches_oracle(lqm, ctx):
    lat, h, v = M.triangular_hubbard(L_super=2)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=3)}
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.02, beta=0.3, tol=0.0, iterations=6)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, **kw)
    assert res.mf.iterations == it == 6
    assert np.max(np.abs(res.rho[(0, 0)] - rho_ref[(0, 0)])) <= RHO_TOL
    assert abs(res.energy - E_ref) <= 1e-9
    assert abs(res.mf.mu - hf_ref.mu) <= 1e-9
    assert abs(res.residual - resid) <= 1e-9


def test_scf_sanitizes_a_non_hermitian_initial_guess(lqm, ctx):
    """Meanfield/selfconsistent.jl:107-113,262-264: a non-Hermitian initial guess is
    made Hermitian (hermitianize!) before the first iteration; the device SCF and the
    oracle then agree as for a Hermitian guess."""
    lat, h, v = M.triangular_hubbard(L_super=2)
    n = h[(0, 0)].shape[0]
    rng = np.random.default_rng(11)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=3) + 0.05 * (rng.normal(size=(n, n))
                                                                             + 1j * rng.normal(size=(n, n)))}
    assert not MF.is_hermitian(rho0)
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.02, beta=0.3, tol=0.0, iterations=4)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, **kw)
    assert np.max(np.abs(res.rho[(0, 0)] - rho_ref[(0, 0)])) <= RHO_TOL
    assert abs(res.energy - E_ref) <= 1e-9 and abs(res.residual - resid) <= 1e-9


def test_hubbard_scf_converges_with_log(lqm, ctx):
    lat, h, v = M.triangular_hubbard(L_super=2)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=5)}
    log = []
    res = lqm.solvehartreefock(h, v, rho0, 0.5, L.regulargrid(6 * 6), T=0.02, beta=0.3, tol=1e-9,
                               iterations=400, log_callback=lambda *a: log.append(a), ctx=ctx)
    assert res.converged and res.residual < 1e-9
    assert len(log) == res.mf.iterations
    # energy decomposition identities at the fixed point (selfconsistent.jl:41-56)
    assert abs(res.energy - (res.mf.eband - res.mf.eH - res.mf.eF)) < 1e-12
    assert abs(res.mf.ekin - (res.mf.eband - 2 * (res.mf.eH + res.mf.eF))) < 1e-12


# ---------------------------------------------------------------- errors (host-side, no device fault)
def test_invalid_inputs_raise(lqm, ctx, c1):
    with pytest.raises(lqm.LQMError) as e:
        lqm.bandmatrix(c1, np.array([[np.nan], [0.0]]), ctx=ctx)
    assert e.value.status == -1
    with pytest.raises(lqm.LQMError):
        lqm.bandmatrix(c1, np.zeros((2, 1)), precision=1, ctx=ctx)
    with pytest.raises(ValueError):
        lqm.bandmatrix(c1, np.zeros((2, 1)), multimode="serial", ctx=ctx)
    bad = {R: m.copy() for R, m in c1.items()}
    bad[(0, 0)][0, 0] = np.inf
    with pytest.raises(lqm.LQMError):
        lqm.DeviceHops(bad, ctx)
    lat, h, v = M.triangular_hubbard(L_super=2)
    with pytest.raises(lqm.LQMError):  # rho keys not closed under L -> -L
        lqm.solvehartreefock(h, v, {(1, 0): np.zeros((8, 8), complex)}, 0.5, np.zeros((2, 1)), ctx=ctx)


def test_fused_bands_dos_rho(lqm, ctx):
    name, h = M.batch_models()[2]
    ks = L.regulargrid(8 * 8)
    w = np.full(ks.shape[1], 1.0 / ks.shape[1])
    b_ref = oracle_bands(h, ks)
    om = np.linspace(b_ref.min(), b_ref.max(), 500)
    rho = {R: None for R in h}
    b, dos, eb = lqm.bands_dos_rho(rho, h, ks, om, 0.05, mu=0.0, T=0.01, ctx=ctx)
    assert rel_band_err(b, b_ref) <= BAND_TOL
    assert np.max(np.abs(dos - K.dos_from_bands(b_ref, om, 0.05))) <= 1e-10 * np.max(dos)
    ref, eb_ref = K.densitymatrix(h, ks, w, 0.0, 0.01, list(h.keys()))
    for R in h:
        assert np.max(np.abs(rho[R] - ref[R])) <= RHO_TOL
    assert abs(eb - eb_ref) <= 1e-9 * max(1.0, abs(eb_ref))


def test_hubbard_scf_anderson_matches_oracle(lqm, ctx):
    """acceleration = :anderson (fixedpoint.jl:64-142, 201-231) on the device against the
    oracle's restatement, 8 iterations with depth 3 (the history fills and rolls over;
    iterations 2+ replay the captured graph).  Bound 1e-8: the two least-squares solves
    (Gram-Schmidt QR here, SVD in the oracle) round differently and the iteration carries
    the difference forward."""
    lat, h, v = M.triangular_hubbard(L_super=2)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=3)}
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.02, beta=0.3, tol=0.0, iterations=8)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, acceleration="anderson", anderson_depth=3, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, acceleration="anderson",
                                                                  anderson_depth=3, **kw)
    assert res.mf.iterations == it == 8
    assert np.max(np.abs(res.rho[(0, 0)] - rho_ref[(0, 0)])) <= 1e-8
    assert abs(res.energy - E_ref) <= 1e-8
    assert abs(res.residual - resid) <= 1e-8 * max(1.0, resid)


def test_commutator_residual_scf_matches_oracle(lqm, ctx):
    """residual_norm = :commutator (selfconsistent.jl:130-166,399-405) through
    lqm_ctx_set_scf_residual: the commutatorresidual case of test/test_meanfield.jl:84-112
    (graphene Hubbard U = 4, antiferromagnetic guess, klin = 9 Wigner-Seitz keys, Anderson
    depth 5) converges below 1e-7 with a residual drop above 1e6, in the oracle's iteration
    count and energy; and lqm_commutator_norm against the oracle on a random rho."""
    _, h, v, rho0 = M.graphene_hubbard(4.0)
    MF.enrichkeys(rho0, 9)
    ks = L.regulargrid(9 * 9)
    kw = dict(T=0.01, beta=1.0, tol=1e-7, iterations=50, acceleration="anderson", anderson_depth=5,
              residual_norm="commutator")
    log = []
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, log_callback=lambda i, e, r, d: log.append(r), **kw)
    rho_ref, E_ref, _, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, **kw)
    assert res.converged and res.residual < 1e-7 and conv
    assert log[0] / log[-1] > 1e6
    assert res.mf.iterations == it
    assert abs(res.energy - E_ref) <= 1e-8

    _, h6 = M.honeycomb_disorder(6)
    rng = np.random.default_rng(5)
    n6 = h6[(0, 0)].shape[0]
    rho = {}
    for R in M.KEYS9:
        X = rng.normal(size=(n6, n6)) + 1j * rng.normal(size=(n6, n6))
        rho[R] = X
    rho = MF.hermitianize(rho)
    ks6 = rng.uniform(-0.5, 0.5, (2, 12))
    c = lqm.commutator_kspace_norm(h6, rho, ks6, ctx=ctx)
    c_ref = MF.commutator_kspace_norm(h6, rho, ks6)
    assert abs(c - c_ref) <= 1e-12 * c_ref


def _jkernel(J1, Jnn):
    # test/test_exchange.jl:14-20
    j0 = np.array([[0.0, J1], [J1, 0.0]], complex)
    jp = np.array([[Jnn, 0.0], [0.0, 0.0]], complex)
    return {(0, 0): j0, (1, 0): jp, (-1, 0): jp.conj().T}


def test_exchange_functional_and_scf_match_oracle(lqm, ctx):
    """J-augmented Hartree-Fock (ExchangeKernel, hartreefock.jl:24-76,298-381) through
    lqm_hartreefock_eval and lqm_scf_hf: hMF and (eH, eF, eJ) for a random complex rho
    with bond keys against the oracle, with each of the Hartree / Fock terms switched off
    too; the analytic dimer limits of test/test_exchange.jl:43-60; and the SCF case of
    test/test_exchange.jl:85-123 (exchange selects the polarized state) in the oracle's
    iterations and energies."""
    siteof, flavorof = [0, 1, 0, 1], [0, 0, 1, 1]
    t, U = 0.1, 1.0
    h = {(0, 0): np.kron(np.eye(2), np.array([[0.0, t], [t, 0.0]], complex))}
    v = {(0, 0): (U * np.ones((4, 4)) - U * np.eye(4)).astype(complex)}
    rng = np.random.default_rng(7)
    r0 = rng.random((4, 4)) + 1j * rng.random((4, 4))
    r1 = rng.random((4, 4)) + 1j * rng.random((4, 4))
    rho = {(0, 0): (r0 + r0.conj().T) / 2, (1, 0): r1, (-1, 0): r1.conj().T}
    for hartree, fock in ((True, True), (False, True), (True, False)):
        ekd = lqm.ExchangeKernel(_jkernel(0.8, 0.35), siteof, flavorof)
        hmf, eH, eF, eJ = lqm.hartreefock_eval(h, v, rho, hartree=hartree, fock=fock, exchange=ekd, ctx=ctx)
        ref = MF.HartreeFock(h, v, hartree=hartree, fock=fock,
                             exchange=MF.ExchangeKernel(_jkernel(0.8, 0.35), siteof, flavorof))(rho)
        assert set(hmf) == set(ref.hMF)
        assert max(np.max(np.abs(hmf[L] - ref.hMF[L])) for L in hmf) <= 1e-12
        assert max(abs(eH - ref.eH), abs(eF - ref.eF), abs(eJ - ref.eJ)) <= 1e-12
    hz = {(0, 0): np.zeros((4, 4), complex)}
    ekd = lqm.ExchangeKernel(_jkernel(0.7, 0.0), siteof, flavorof)
    _, _, _, eJ = lqm.hartreefock_eval(hz, hz, {(0, 0): np.diag([1.0, 1, 0, 0]).astype(complex)}, exchange=ekd,
                                       ctx=ctx)
    assert abs(eJ + 0.7) < 1e-12
    _, _, _, eJ = lqm.hartreefock_eval(hz, hz, {(0, 0): 0.5 * np.eye(4, dtype=complex)}, exchange=ekd, ctx=ctx)
    assert abs(eJ + 0.35) < 1e-12
    with pytest.raises(lqm.LQMError):
        lqm.hartreefock_eval(hz, hz, rho, exchange=lqm.ExchangeKernel(
            {(0, 0): np.array([[0.5, 0], [0, 0]], complex)}, siteof, flavorof), ctx=ctx)

    ks = L.regulargrid(8 * 8)
    Es = {}
    for label, occs, J in (("pol_J", [0.9, 0.9, 0.1, 0.1], 0.4), ("unp_J", [0.5] * 4, 0.4),
                           ("pol_0", [0.9, 0.9, 0.1, 0.1], None), ("unp_0", [0.5] * 4, None)):
        rho0 = {(0, 0): np.diag(occs).astype(complex)}
        kw = dict(T=0.02, beta=0.5, tol=1e-9, iterations=600)
        res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, **kw,
                                   exchange=lqm.ExchangeKernel(_jkernel(J, 0.0), siteof, flavorof) if J else None)
        _, E_ref, hf_ref, conv, _, it = MF.solvehartreefock(
            h, v, rho0, 0.5, ks, **kw, exchange=MF.ExchangeKernel(_jkernel(J, 0.0), siteof, flavorof) if J else None)
        assert res.converged and conv
        assert abs(res.energy - (res.mf.ekin + res.mf.eH + res.mf.eF + res.mf.eJ)) <= 1e-6 + 1e-8 * abs(res.energy)
        assert abs(res.energy - E_ref) <= 1e-8 and abs(res.mf.eJ - hf_ref.eJ) <= 1e-8
        assert abs(res.mf.iterations - it) <= 1
        Es[label] = res.energy
    assert (Es["unp_J"] - Es["pol_J"]) - (Es["unp_0"] - Es["pol_0"]) > 0.3 * 0.4


def test_bdg_paths_match_oracle(lqm, ctx):
    """Nambu (BdG) Hamiltonians through lqm_bdg_densitymatrix, lqm_bdg_filling and
    lqm_bdg_chemicalpotential: the checks of test/test_superconductivity.jl (+-E pairs,
    the 2 Delta gap at the Dirac point, the BdG kinetic energy -3 at Gamma, filling 1/2
    with weak pairing) on the device, and parity with the oracle for the disordered
    honeycomb 3x3 cell (n = 36, BdG order 72) with complex onsite and bond pairing."""
    from oracle import bdg as BDG
    lat = L.honeycomb()
    h = M.nearestneighbor(lat, -1.0)
    H = M.bdg_operator(h)
    b, _ = lqm.bandmatrix(H, np.array([[0.1, 0.3, 0.0], [0.2, -0.1, 0.0]]), ctx=ctx)
    assert np.max(np.abs(b + b[::-1, :])) < 1e-10
    Hs = M.bdg_operator(h, {(0, 0): 0.25 * np.eye(2, dtype=complex)})
    b, _ = lqm.bandmatrix(Hs, np.array([[1 / 3], [-1 / 3]]), ctx=ctx)
    assert abs(b[2, 0] - 0.25) < 1e-10 and abs(b[1, 0] + 0.25) < 1e-10
    rho = {R: None for R in H}
    e = lqm.bdg_getdensitymatrix(rho, H, np.zeros((2, 1)), mu=0.0, T=1e-6, ctx=ctx)
    assert abs(e + 3.0) < 1e-3
    Hw = M.bdg_operator(h, {(0, 0): 0.05 * np.eye(2, dtype=complex)})
    assert abs(lqm.bdg_filling(Hw, L.regulargrid(12 * 12), 0.0, T=0.05, ctx=ctx) - 0.5) < 5e-3

    _, h3 = M.honeycomb_disorder(3)
    n = h3[(0, 0)].shape[0]
    rng = np.random.default_rng(9)
    D0 = 0.1 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    D1 = 0.05 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    delta = {(0, 0): D0 - D0.T, (1, 0): D1, (-1, 0): -D1.T}
    HB = M.bdg_operator(h3, delta)
    assert HB.keys() == BDG.bdg_operator(h3, delta).keys()
    ks = rng.uniform(-0.5, 0.5, (2, 10))
    w = np.full(10, 0.1)
    rho = {R: None for R in M.KEYS9}
    e = lqm.bdg_getdensitymatrix(rho, HB, ks, mu=0.3, T=0.02, ctx=ctx)
    rref, eref = BDG.bdg_densitymatrix(BDG.bdg_operator(h3, delta), ks, w, 0.3, 0.02, M.KEYS9)
    assert max(np.max(np.abs(rho[R] - rref[R])) for R in M.KEYS9) <= 1e-9
    assert abs(e - eref) <= 1e-10 * max(1.0, abs(eref))
    f = lqm.bdg_filling(HB, ks, 0.3, T=0.05, ctx=ctx)
    assert abs(f - BDG.bdg_filling(HB, ks, 0.3, T=0.05)) <= 1e-12
    mu = lqm.bdg_chemicalpotential(HB, ks, 0.45, T=0.05, ctx=ctx)
    mu_ref = BDG.bdg_chemicalpotential(HB, ks, 0.45, T=0.05)
    assert abs(mu - mu_ref) <= 1e-9
    assert abs(lqm.bdg_filling(HB, ks, mu, T=0.05, ctx=ctx) - 0.45) <= 1e-10


def test_bdg_scf_matches_oracle(lqm, ctx):
    """HartreeFockBDG SCF (Superconductivity/hartreefock.jl:5-159 in the SCF loop, BdG mu and
    rho) through lqm_scf_hf_bdg against the oracle: spinful graphene with attractive Hubbard
    U = -3 (sigma_x mode) from a small singlet pairing guess, 6 iterations of linear mixing
    (beta = 0.5, T = 0.05) on a 6 x 6 grid; then a superconducting solution holds eP < 0."""
    from oracle import bdg as BDG
    lat = L.honeycomb()
    h = M.graphene(lat, spin=True)
    v = M.hubbard_v(lat, U=-3.0)
    r0 = np.zeros((8, 8), complex)
    r0[:4, :4] = 0.5 * np.eye(4)
    r0[4:, 4:] = 0.5 * np.eye(4)
    D = np.zeros((4, 4), complex)
    for i in range(2):
        D[2 * i, 2 * i + 1], D[2 * i + 1, 2 * i] = 0.1, -0.1
    r0[:4, 4:] = D
    r0[4:, :4] = D.conj().T
    rho = {R: np.zeros((8, 8), complex) for R in h}
    rho[(0, 0)] = r0
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.05, beta=0.5, tol=0.0, iterations=6)
    res = lqm.solvehartreefock_bdg(h, v, rho, 0.5, ks, ctx=ctx, **kw)
    rho_ref, E_ref, hf_ref, _, resid, it = BDG.solvehartreefock_bdg(h, v, rho, 0.5, ks, **kw)
    assert res.mf.iterations == it == 6
    assert abs(res.mf.mu - hf_ref.mu) <= 1e-9
    assert abs(res.energy - E_ref) <= 1e-9 and abs(res.mf.eP - hf_ref.eP) <= 1e-9
    assert max(np.max(np.abs(res.rho[R] - rho_ref[R])) for R in rho) <= 1e-9
    assert abs(res.residual - resid) <= 1e-9
    assert res.mf.eP < -1e-3


def test_bdg_scf_anderson_and_commutator_match_oracle(lqm, ctx):
    """lqm_scf_hf_bdg with Anderson acceleration (depth 3, the Nambu iterate projected
    Hermitian) and with the commutator residual ||[HB, rho]|| against the oracle, 6
    iterations of the attractive-U graphene case.  Bound 1e-8 for Anderson (its
    least-squares solves round differently)."""
    from oracle import bdg as BDG
    lat = L.honeycomb()
    h = M.graphene(lat, spin=True)
    v = M.hubbard_v(lat, U=-3.0)
    r0 = np.zeros((8, 8), complex)
    r0[:4, :4] = 0.5 * np.eye(4)
    r0[4:, 4:] = 0.5 * np.eye(4)
    for i in range(2):
        r0[2 * i, 4 + 2 * i + 1], r0[2 * i + 1, 4 + 2 * i] = 0.1, -0.1
    r0[4:, :4] = r0[:4, 4:].conj().T
    rho = {R: np.zeros((8, 8), complex) for R in h}
    rho[(0, 0)] = r0
    ks = L.regulargrid(6 * 6)
    for extra, tolr in ((dict(acceleration="anderson", anderson_depth=3), 1e-8),
                        (dict(residual_norm="commutator"), 1e-9)):
        kw = dict(T=0.05, beta=0.5, tol=0.0, iterations=6, **extra)
        res = lqm.solvehartreefock_bdg(h, v, rho, 0.5, ks, ctx=ctx, **kw)
        rho_ref, E_ref, hf_ref, _, resid, it = BDG.solvehartreefock_bdg(h, v, rho, 0.5, ks, **kw)
        assert res.mf.iterations == it == 6
        assert abs(res.energy - E_ref) <= tolr
        assert max(np.max(np.abs(res.rho[R] - rho_ref[R])) for R in rho) <= tolr
        assert abs(res.residual - resid) <= tolr * max(1.0, resid)


def test_bdg_scf_anderson_converges_like_oracle(lqm, ctx):
    """The accelerated BdG SCF converges: Anderson (depth 3) on the attractive-U
    graphene case reaches the relative residual 1e-8 (the oracle takes 18 iterations,
    plain linear mixing 90), in the oracle's iteration count, at the oracle's fixed
    point (pairing field, energy and mu to 1e-8)."""
    from oracle import bdg as BDG
    lat = L.honeycomb()
    h = M.graphene(lat, spin=True)
    v = M.hubbard_v(lat, U=-3.0)
    r0 = np.zeros((8, 8), complex)
    r0[:4, :4] = 0.5 * np.eye(4)
    r0[4:, 4:] = 0.5 * np.eye(4)
    for i in range(2):
        r0[2 * i, 4 + 2 * i + 1], r0[2 * i + 1, 4 + 2 * i] = 0.1, -0.1
    r0[4:, :4] = r0[:4, 4:].conj().T
    rho = {R: np.zeros((8, 8), complex) for R in h}
    rho[(0, 0)] = r0
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.05, beta=0.5, tol=1e-8, iterations=100, acceleration="anderson", anderson_depth=3)
    res = lqm.solvehartreefock_bdg(h, v, rho, 0.5, ks, ctx=ctx, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = BDG.solvehartreefock_bdg(h, v, rho, 0.5, ks, **kw)
    assert conv and it < 100
    assert res.residual <= 1e-8
    assert abs(res.mf.iterations - it) <= 1
    assert abs(res.energy - E_ref) <= 1e-8
    assert max(np.max(np.abs(res.rho[R] - rho_ref[R])) for R in rho) <= 1e-8
    assert abs(res.mf.mu - hf_ref.mu) <= 1e-8


def test_eigh_block_sizes_and_autotuner(lqm):
    """Every block size the autotuner may choose for the batched models (n = 8, 24, 96)
    gives the oracle's bands, eigenvectors and rho_L; the autotuner then keeps one of
    them, and a repeated call with that block size is bit-identical."""
    c = lqm.Context(0, timeout=600)
    try:
        rng = np.random.default_rng(21)
        ks = rng.uniform(-0.5, 0.5, (2, 24))
        w = np.full(24, 1 / 24)
        for name, h in M.batch_models():
            n = h[(0, 0)].shape[0]
            base = 32 if n <= 16 else (64 if n <= 32 else (128 if n < 64 else 384))
            cands = [nt for nt in (32, 64, 128, 256, 384, 512) if max(32, base // 2) <= nt <= max(4 * base, 512)]
            bref, _ = K.bandmatrix(h, ks)
            rref, _ = K.densitymatrix(h, ks, w, 0.0, 0.01, list(h.keys()))
            for nt in cands:
                c.set_eigh_threads(n, nt)
                b, U = lqm.bandmatrix(h, ks, want_vectors=True, ctx=c)
                assert rel_band_err(b, bref) <= BAND_TOL, (name, nt)
                for j in range(ks.shape[1]):
                    Hk = K.fouriersum(h, ks[:, j])
                    assert np.max(np.abs(Hk @ U[:, :, j] - U[:, :, j] * b[:, j])) <= 1e-10 * max(1.0, np.ptp(bref))
                rho = {R: None for R in h}
                lqm.getdensitymatrix(rho, h, ks, mu=0.0, T=0.01, ctx=c)
                assert max(np.max(np.abs(rho[R] - rref[R])) for R in h) <= RHO_TOL, (name, nt)
            best, ms, table = lqm.autotune_eigh(h, rng.uniform(-0.5, 0.5, (2, 4096)), ctx=c)
            assert best in cands and set(table) == set(cands) and ms == min(table.values())
            rho1, rho2 = {R: None for R in h}, {R: None for R in h}
            lqm.getdensitymatrix(rho1, h, ks, mu=0.0, T=0.01, ctx=c)
            lqm.getdensitymatrix(rho2, h, ks, mu=0.0, T=0.01, ctx=c)
            assert all(np.array_equal(rho1[R], rho2[R]) for R in h)
            c.set_eigh_threads(n, 0)
    finally:
        c.close()


def test_hard_hermitian_inputs_both_paths(lqm):
    """The hard Hermitian inputs of the emulation suite (zero reflectors, whole
    degenerate clusters, pairs split by 1e-13, zero rows, rank one, scales 1e+-150)
    through the C-ABI on the one-CTA kernel and on the blocked path."""
    from test_emulation import _hard_hermitian
    cases = _hard_hermitian()
    ks = np.zeros((2, 1))
    for blocked in (False, True):
        c = lqm.Context(0, timeout=600)
        try:
            if blocked:
                c.set_blocked_min_n(1)
            for name, Hk in cases:
                b, U = lqm.bandmatrix({(0, 0): Hk}, ks, want_vectors=True, ctx=c)
                n = Hk.shape[0]
                ref = K.eigh_upper(Hk, vectors=False)
                scale = max(np.max(np.abs(ref)), np.finfo(float).tiny)
                Uk = U[:, :, 0]
                assert np.all(np.isfinite(Uk)), (name, blocked)
                assert np.max(np.abs(b[:, 0] - ref)) <= 1e-12 * scale, (name, blocked)
                assert np.max(np.abs(Uk.conj().T @ Uk - np.eye(n))) <= 1e-12, (name, blocked)
                assert np.max(np.abs(Hk @ Uk - Uk * b[:, 0])) <= 1e-12 * scale, (name, blocked)
        finally:
            c.close()


def test_parallelism_pin_filling_and_energy(lqm, ctx):
    """test/test_parallelism.jl:49-106 on the CUDA path: graphene nearest neighbour,
    mu = 0, T = 0.05, 12^2 and 8^2 grids: filling tr(rho_0)/2 and band energy equal
    the oracle's serial k-loop to 1e-10, three runs give identical results, and the
    band energy is not lost (nonzero)."""
    h = M.nearestneighbor(L.honeycomb(), -1.0)
    for nk_lin in (12, 8):
        ks = L.regulargrid(nk_lin * nk_lin)
        w = np.full(ks.shape[1], 1.0 / ks.shape[1])
        ref, eb_ref = K.densitymatrix(h, ks, w, 0.0, 0.05, list(h.keys()))
        f_ref = np.real(np.trace(ref[(0, 0)])) / 2
        runs = []
        for _ in range(3):
            rho = {R: None for R in h}
            eb = lqm.getdensitymatrix(rho, h, ks, mu=0.0, T=0.05, ctx=ctx)
            runs.append((np.real(np.trace(rho[(0, 0)])) / 2, eb))
        assert runs[0] == runs[1] == runs[2]
        f, eb = runs[0]
        assert abs(f - f_ref) <= 1e-10 and abs(eb - eb_ref) <= 1e-10 and eb != 0.0


def test_scf_interaction_range_beyond_hopping_range(lqm, ctx):
    """test/test_meanfield.jl:256-278 through the device SCF: onsite-only h, a Hubbard
    interaction on 9 neighbour cells (a = 1.8), antiferromagnetic start; 3 iterations
    match the oracle's (the mean field carries the keys of v that h lacks)."""
    lat = L.honeycomb()
    h = {(0, 0): np.diag([0.3, 0.3, -0.3, -0.3]).astype(complex)}
    nbrs = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, -1), (1, -1), (-1, 1)]
    v = M.hubbard_v(lat, U=2.0, a=1.8, neighbors=nbrs)
    rho0 = {R: np.zeros((4, 4), complex) for R in v}
    rho0[(0, 0)] = M.antiferro_density(lat)
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.05, beta=0.3, tol=0.0, iterations=3)
    res = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, **kw)
    rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, **kw)
    for R in rho_ref:
        assert np.max(np.abs(res.rho[R] - rho_ref[R])) <= RHO_TOL, R
    assert abs(res.energy - E_ref) <= 1e-9 and abs(res.residual - resid) <= 1e-9


def test_host_wait_limit_reports_timeout_and_context_recovers(lqm):
    """Failure handling without a GPU fault: the host waits for device work by
    polling with a per-context limit (lqm_ctx_set_timeout).  A limit far below the
    work's duration ends the call with LQM_ETIMEOUT while the kernel runs to
    completion on its own; with the limit restored, the same context serves the
    next call correctly.  (Device-pointer entry point: its only wait is the poll.)"""
    import torch
    c = lqm.Context(0, timeout=600)
    try:
        dev = torch.device("cuda", 0)
        h = M.batch_models()[2][1]  # n = 96: 8192 k-points are tens of ms of device work
        ks = np.random.default_rng(2).random((2, 8192))
        Hd = lqm.DeviceHops(h, c)
        d_ks = torch.from_numpy(np.ascontiguousarray(ks.T)).to(dev)
        d_b = torch.zeros(ks.shape[1], Hd.n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()  # the library runs on its own stream: inputs complete first

        def call():
            return lqm.lib().lqm_bandmatrix_dev(c.handle, Hd.handle, ks.shape[1], lqm._ptr(d_ks), 0, 0,
                                                lqm._ptr(d_b), None)
        c.check(call())  # plans and workspaces exist before the limit is lowered
        c.check(lqm.lib().lqm_ctx_set_timeout(c.handle, 1e-6))
        assert call() == -4
        c.check(lqm.lib().lqm_ctx_set_timeout(c.handle, 600.0))
        c.check(call())  # queued behind the first kernel on the context's stream; rewrites every band
        b = d_b.cpu().numpy().T
        assert rel_band_err(b[:, :64], oracle_bands(h, ks[:, :64])) <= BAND_TOL
        Hd.free()
    finally:
        c.close()
