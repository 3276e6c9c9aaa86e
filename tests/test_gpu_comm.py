"""The multi-GPU sharding code path on one GPU: a one-rank NCCL communicator set on
a context makes lqm_densitymatrix, lqm_bands_dos_rho, lqm_bandmatrix,
lqm_chemicalpotential, lqm_dos and lqm_scf_hf take their sharded branches (the
share of the k list, ncclAllReduce of rho_L and the band energy, ncclBroadcast of
the bands and vectors, the SCF without graph replay), whose collectives are then
copies.  The results must equal those of a context without a communicator.  (Two
or more ranks need one GPU each; the decomposition itself is checked against the
serial oracle on two gloo ranks in test_multirank_cpu.py.)"""
import numpy as np
import pytest

from lqm_workloads import lattice as L
from lqm_workloads import models as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cctx(lqm):
    c = lqm.Context(0, timeout=300)
    c.set_comm(1, 0, lqm.comm_unique_id())
    assert c.comm() == (1, 0)
    yield c
    c.set_comm(1, 0)
    assert c.comm() == (1, 0)
    c.close()


@pytest.mark.parametrize("which", [1, 2])
def test_one_rank_communicator_matches_plain_context(lqm, ctx, cctx, which):
    """n = 24 (one-CTA path) and n = 144 (blocked path)."""
    h = M.batch_models()[1][1] if which == 1 else M.honeycomb_disorder()[1]
    ks = L.regulargrid(7 * 7)
    keys = list(h.keys())
    r1, r2 = {R: None for R in keys}, {R: None for R in keys}
    e1 = lqm.getdensitymatrix(r1, h, ks, mu=0.0, T=0.01, ctx=ctx)
    e2 = lqm.getdensitymatrix(r2, h, ks, mu=0.0, T=0.01, ctx=cctx)
    assert e1 == e2 and all(np.array_equal(r1[R], r2[R]) for R in keys)
    b1, U1 = lqm.bandmatrix(h, ks, want_vectors=True, ctx=ctx)
    b2, U2 = lqm.bandmatrix(h, ks, want_vectors=True, ctx=cctx)
    assert np.array_equal(b1, b2) and np.array_equal(U1, U2)
    assert lqm.chemicalpotential(h, ks, 0.4, T=0.05, ctx=ctx) == lqm.chemicalpotential(h, ks, 0.4, T=0.05, ctx=cctx)
    om = np.linspace(b1.min(), b1.max(), 40)
    assert np.array_equal(lqm.getdos(h, om, ks, 0.05, ctx=ctx), lqm.getdos(h, om, ks, 0.05, ctx=cctx))
    f1, f2 = {R: None for R in keys}, {R: None for R in keys}
    o1 = lqm.bands_dos_rho(f1, h, ks, om, 0.05, mu=0.0, T=0.01, ctx=ctx)
    o2 = lqm.bands_dos_rho(f2, h, ks, om, 0.05, mu=0.0, T=0.01, ctx=cctx)
    assert np.array_equal(o1[0], o2[0]) and np.array_equal(o1[1], o2[1]) and o1[2] == o2[2]
    assert all(np.array_equal(f1[R], f2[R]) for R in keys)


def test_one_rank_communicator_scf(lqm, ctx, cctx):
    lat, h, v = M.triangular_hubbard(L_super=3)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=2)}
    ks = L.regulargrid(6 * 6)
    kw = dict(T=0.02, beta=0.3, tol=0.0, iterations=6)
    a = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, **kw)
    b = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=cctx, **kw)
    assert np.max(np.abs(a.rho[(0, 0)] - b.rho[(0, 0)])) <= 1e-14
    assert abs(a.energy - b.energy) <= 1e-12 and abs(a.mf.mu - b.mf.mu) <= 1e-14
    c = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=cctx, residual_norm="commutator", **kw)
    d = lqm.solvehartreefock(h, v, rho0, 0.5, ks, ctx=ctx, residual_norm="commutator", **kw)
    assert abs(c.residual - d.residual) <= 1e-12
