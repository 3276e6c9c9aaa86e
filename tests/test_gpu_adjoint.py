"""Reverse-mode derivatives through the C-ABI (lqm_densitymatrix_vjp, lqm_bands_vjp)
against the oracle adjoint and against central finite differences of the CUDA
forward map.  Tolerances: 1e-10 of the largest cotangent entry against the oracle
(FP64 both sides), 1e-6 relative against finite differences (step 1e-6)."""
import numpy as np
import pytest

from oracle import adjoint as AD
from oracle import kspace as K
from lqm_workloads import lattice as L
from lqm_workloads import models as M

pytestmark = pytest.mark.gpu


def max_err(A, B):
    scale = max(max(np.max(np.abs(B[R])) for R in B), 1e-300)
    return max(np.max(np.abs(A[R] - B[R])) for R in B) / scale


@pytest.fixture(scope="module")
def bctx(lqm):
    c = lqm.Context(0, timeout=900)
    c.set_blocked_min_n(1)
    yield c
    c.close()


def _cases():
    out = M.batch_models()
    out.append(("honeycomb144", M.honeycomb_disorder()[1]))
    return out


@pytest.mark.parametrize("blocked", [False, True], ids=["one-cta", "blocked"])
def test_densitymatrix_vjp_matches_oracle(lqm, ctx, bctx, blocked):
    c = bctx if blocked else ctx
    rng = np.random.default_rng(21)
    for name, h in _cases():
        ks = rng.random((2, 6))
        w = rng.random(6)
        w /= w.sum()
        n = h[(0, 0)].shape[0]
        Gbar = {L_: rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) for L_ in [(0, 0), (1, 0), (0, -1)]}
        for T in (0.05, 0.0):
            got = lqm.densitymatrix_vjp(h, ks, Gbar, kweights=w, mu=0.1, T=T, ctx=c)
            ref = AD.densitymatrix_vjp(h, ks, w, 0.1, T, Gbar)
            assert max_err(got, ref) <= 1e-10, (name, T)


def test_densitymatrix_vjp_finite_differences_on_gpu(lqm, ctx):
    """The CUDA adjoint against central differences of the CUDA forward map."""
    h = M.batch_models()[1][1]  # kagome, n = 24
    rng = np.random.default_rng(5)
    ks = L.regulargrid(5 * 5)
    keys = list(h.keys())
    n = h[(0, 0)].shape[0]
    Gbar = {L_: rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) for L_ in keys}
    mu, T = 0.05, 0.05
    Hbar = lqm.densitymatrix_vjp(h, ks, Gbar, mu=mu, T=T, ctx=ctx)
    dH = AD.hermitian_direction(h, rng)

    def loss(hh):
        rho = {L_: None for L_ in keys}
        lqm.getdensitymatrix(rho, hh, ks, mu=mu, T=T, ctx=ctx)
        return AD.pairing(Gbar, rho)

    step = 1e-6
    fd = (loss({R: h[R] + step * dH[R] for R in h}) - loss({R: h[R] - step * dH[R] for R in h})) / (2 * step)
    an = AD.pairing(Hbar, dH)
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


@pytest.mark.parametrize("blocked", [False, True], ids=["one-cta", "blocked"])
def test_bands_vjp_matches_oracle(lqm, ctx, bctx, blocked):
    c = bctx if blocked else ctx
    rng = np.random.default_rng(3)
    for name, h in M.batch_models():
        n = h[(0, 0)].shape[0]
        ks = rng.random((2, 5))
        # equal weights on the spin-degenerate pairs keep the loss differentiable
        eb = np.repeat(rng.normal(size=(n // 2, 5)), 2, axis=0)
        got = lqm.bands_vjp(h, ks, eb, ctx=c)
        ref = AD.bands_vjp(h, ks, eb)
        assert max_err(got, ref) <= 1e-9, name


def test_densitymatrix_vjp_large_n(lqm, ctx):
    """Twisted bilayer m=10 (n = 1324, blocked path) on two k-points."""
    _, h = M.tbg_slater_koster(10)
    n = h[(0, 0)].shape[0]
    rng = np.random.default_rng(2)
    ks = np.array([[0.1, 0.37], [0.2, -0.11]])
    w = np.array([0.5, 0.5])
    Gbar = {(0, 0): rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))}
    got = lqm.densitymatrix_vjp(h, ks, Gbar, kweights=w, mu=0.0, T=0.02, ctx=ctx)
    ref = AD.densitymatrix_vjp(h, ks, w, 0.0, 0.02, Gbar)
    assert max_err(got, ref) <= 1e-9
