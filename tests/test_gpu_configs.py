"""Parity at the workload configurations' own sizes, through the C ABI.

* the Hartree-Fock SCF of the triangular Hubbard model at its full size
  (n = 72, 36 x 36 k-points, T = 0.02, linear mixing beta = 0.3) run to the
  relative residual 1e-9, against the oracle's converged run committed by
  tests/golden/make_scf_c4.py (src/modules/Meanfield/selfconsistent.jl:256-336,
  fixedpoint.jl:143-178);
* the twisted bilayer m = 15 (n = 2884): bands, eigenpairs and rho_L on two
  k-points, and one Hartree-Fock iteration with the screened Coulomb
  interaction, against the oracle run live;
* the SparseHops upload (every reference Hops with n > MAX_DENSE = 500 arrives
  as SparseMatrixCSC, src/modules/TightBinding/types.jl:102-103,272): the
  n = 1324 bilayer uploaded from 1-based CSC blocks gives bit-identical H(k) and
  bands to the dense upload, and malformed CSC input is rejected on the host.
"""
import ctypes
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


def oracle_threads():
    """The oracle's LAPACK calls at n = 2884 take seconds per k-point on one core;
    let them use the host's cores (the suite pins BLAS to one thread otherwise)."""
    from threadpoolctl import threadpool_limits
    return threadpool_limits(limits=max(1, min(32, os.cpu_count() or 1)))


def test_c4_hubbard_scf_converged_matches_oracle(lqm, ctx):
    """Triangular Hubbard HF at n = 72 on 36 x 36 k-points, converged to 1e-9."""
    g = np.load(os.path.join(GOLD, "scf_c4_oracle.npz"))
    assert bool(g["converged"])
    lat, h, v = M.triangular_hubbard(L_super=int(g["L_super"]))
    assert h[(0, 0)].shape[0] == 72
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=int(g["seed"]))}
    ks = L.regulargrid(int(g["nk_side"]) ** 2)
    res = lqm.solvehartreefock(h, v, rho0, float(g["filling"]), ks, T=float(g["T"]), beta=float(g["beta"]),
                               tol=float(g["tol"]), iterations=int(g["maxiter"]), ctx=ctx)
    assert res.converged and res.residual < 1e-9
    # the same trajectory: the device SCF stops within a step of the oracle's count
    assert abs(res.mf.iterations - int(g["iterations"])) <= 1
    assert np.max(np.abs(res.rho[(0, 0)] - g["rho0"])) <= RHO_TOL
    assert abs(res.mf.mu - float(g["mu"])) <= 1e-9
    assert abs(res.energy - float(g["E"])) <= 1e-9 * max(1.0, abs(float(g["E"])))
    assert abs(res.mf.eH - float(g["eH"])) <= 1e-9 * max(1.0, abs(float(g["eH"])))
    assert abs(res.mf.eF - float(g["eF"])) <= 1e-9 * max(1.0, abs(float(g["eF"])))


@pytest.fixture(scope="module")
def tbg15():
    return M.tbg_screened_hf(15)


def test_c5_tbg_2884_bands_vectors_rho(lqm, ctx, tbg15):
    """Twisted bilayer m = 15 (n = 2884) on two k-points: bands to 1e-10 of the
    spectral width, orthonormal eigenpairs, rho_L (all 7 keys of H) to 1e-9."""
    _, h, _ = tbg15
    n = h[(0, 0)].shape[0]
    assert n == 2884
    ks = np.array([[0.0, 0.41], [0.0, 0.17]])
    b, U = lqm.bandmatrix(h, ks, want_vectors=True, ctx=ctx)
    w = np.full(ks.shape[1], 0.5)
    keys = list(h.keys())
    rho = {R: None for R in keys}
    eb = lqm.getdensitymatrix(rho, h, ks, kweights=w, mu=0.0, T=0.01, ctx=ctx)
    with oracle_threads():
        ref_b, _ = K.bandmatrix(h, ks)
        rref, ebref = K.densitymatrix(h, ks, w, 0.0, 0.01, keys)
    assert rel_band_err(b, ref_b) <= BAND_TOL
    for j in range(ks.shape[1]):
        Hk = K.fouriersum(h, ks[:, j])
        Uj = U[:, :, j]
        assert np.max(np.abs(Uj.conj().T @ Uj - np.eye(n))) < 1e-11
        assert np.max(np.abs(Hk @ Uj - Uj * b[:, j])) < 1e-10
    assert max(np.max(np.abs(rho[R] - rref[R])) for R in keys) <= RHO_TOL
    assert abs(eb - ebref) <= 1e-9 * max(1.0, abs(ebref))


def test_c5_tbg_2884_one_hf_iteration(lqm, ctx, tbg15):
    """One Hartree-Fock iteration of the n = 2884 bilayer with the screened Coulomb
    interaction (9 keys) on two k-points: mean field, mu (T = 0.05 bisection), the
    mixed rho_L, the energies."""
    _, h, v = tbg15
    n = h[(0, 0)].shape[0]
    rng = np.random.default_rng(11)
    X = rng.normal(size=(n, n)) * 0.01
    r0 = {R: np.zeros((n, n), complex) for R in v}
    r0[(0, 0)] = 0.5 * np.eye(n) + (X + X.T)
    ks = np.array([[0.0, 1.0 / 3.0], [0.25, 1.0 / 3.0]])
    kw = dict(T=0.05, beta=0.3, tol=0.0, iterations=1)
    res = lqm.solvehartreefock(h, v, r0, 0.5, ks, ctx=ctx, **kw)
    with oracle_threads():
        rho_ref, E_ref, hf_ref, conv, resid, it = MF.solvehartreefock(h, v, r0, 0.5, ks, **kw)
    assert res.mf.iterations == it == 1
    assert max(np.max(np.abs(res.rho[R] - rho_ref[R])) for R in v) <= RHO_TOL
    assert abs(res.mf.mu - hf_ref.mu) <= 1e-9
    assert abs(res.energy - E_ref) <= 1e-9 * max(1.0, abs(E_ref))
    assert abs(res.residual - resid) <= 1e-9


def test_csc_upload_bit_identical_to_dense(lqm, ctx):
    """The n = 1324 bilayer from 1-based SparseMatrixCSC blocks: the same device
    blocks, H(k) and bands as the dense upload, bit for bit."""
    import scipy.sparse as sp
    _, h = M.tbg_slater_koster(10)
    n = h[(0, 0)].shape[0]
    assert n == 1324
    hs = {R: sp.csc_matrix(Mx) for R, Mx in h.items()}
    fill = sum(m.nnz for m in hs.values()) / (n * n * len(hs))
    assert fill < 0.2
    Hd = lqm.DeviceHops(h, ctx)
    Hs = lqm.DeviceHops(hs, ctx)
    ks = np.array([[0.0, 0.23, 1 / 3], [0.0, 0.61, -1 / 3]])
    Bd = lqm.bloch(Hd, ks, ctx=ctx)
    Bs = lqm.bloch(Hs, ks, ctx=ctx)
    assert np.array_equal(Bd, Bs)
    bd, _ = lqm.bandmatrix(Hd, ks, ctx=ctx)
    bs, _ = lqm.bandmatrix(Hs, ks, ctx=ctx)
    assert np.array_equal(bd, bs)
    # repeated (row, column) entries are summed, as a dense accumulation would
    c = hs[(0, 0)]
    ind, dat, ptr = [], [], [0]
    for j in range(n):
        idx = c.indices[c.indptr[j]:c.indptr[j + 1]]
        val = c.data[c.indptr[j]:c.indptr[j + 1]]
        ind += [idx, idx]
        dat += [0.25 * val, 0.75 * val]
        ptr.append(ptr[-1] + 2 * idx.size)
    dup = sp.csc_matrix((np.concatenate(dat), np.concatenate(ind), np.array(ptr)), shape=(n, n))
    assert dup.data.size == 2 * c.nnz  # both copies of every entry are stored
    hdup = dict(hs)
    hdup[(0, 0)] = dup
    b2, _ = lqm.bandmatrix(lqm.DeviceHops(hdup, ctx), ks[:, :1], ctx=ctx)
    assert rel_band_err(b2, bd[:, :1]) <= 1e-13
    Hd.free()
    Hs.free()


def _csc_call(lqm, ctx, n, colptr, rowval, nzval, nnz):
    keys = np.zeros((2, 1), dtype=np.int64, order="F")
    arr = ctypes.c_void_p * 1
    out = ctypes.c_void_p()
    nnz_arr = np.array([nnz], dtype=np.int64)
    cp, rv, nz = arr(colptr.ctypes.data), arr(rowval.ctypes.data), arr(nzval.ctypes.data)
    st = lqm._lib.lqm_hops_upload_csc(ctx.handle, n, 1, 2, keys.ctypes.data, ctypes.cast(cp, ctypes.c_void_p),
                                      ctypes.cast(rv, ctypes.c_void_p), ctypes.cast(nz, ctypes.c_void_p),
                                      nnz_arr.ctypes.data, ctypes.byref(out))
    if st == 0:
        lqm._lib.lqm_hops_free(ctx.handle, out)
    return st


def test_csc_upload_rejects_malformed_input(lqm, ctx):
    """Host-side checks: colptr must start at 1, not decrease and end within nnz; rows in 1..n;
    values finite.  Each failure is LQM_EINVAL before any device work."""
    n = 4
    colptr = np.array([1, 2, 3, 4, 5], dtype=np.int64)
    rowval = np.array([1, 2, 3, 4], dtype=np.int64)
    nzval = np.ones(4, dtype=np.complex128)
    assert _csc_call(lqm, ctx, n, colptr, rowval, nzval, 4) == 0
    assert _csc_call(lqm, ctx, n, colptr, rowval, nzval, 3) == -1        # colptr ends past nnz
    assert _csc_call(lqm, ctx, n, colptr - 1, rowval, nzval, 4) == -1    # 0-based colptr
    assert _csc_call(lqm, ctx, n, np.array([1, 3, 2, 4, 5], dtype=np.int64), rowval, nzval, 4) == -1
    assert _csc_call(lqm, ctx, n, colptr, np.array([1, 2, 5, 4], dtype=np.int64), nzval, 4) == -1
    bad = nzval.copy()
    bad[2] = np.nan
    assert _csc_call(lqm, ctx, n, colptr, rowval, bad, 4) == -1
