"""CPU check of the eigensolver's team code (host build of lqm_eigh.cuh) against the oracle.

The CUDA kernel and this host build share every line of bloch_build / hetrd_lower /
dc_solve / backtransform; only the team shape differs (one thread, one lane here).
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import kspace as K
from lqm_workloads import lattice as L
from lqm_workloads import models as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P = ctypes.c_void_p


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    out = tmp_path_factory.mktemp("emul") / "libemul.so"
    src = os.path.join(ROOT, "tests", "native", "eigh_emul.cpp")
    inc = os.path.join(ROOT, "latticeqm.jl_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I", inc, src, "-o", str(out)],
                   check=True)
    return ctypes.CDLL(str(out))


def pack(h):
    keys = np.asfortranarray(np.array(list(h.keys()), dtype=np.int64).T)
    blocks = np.asfortranarray(np.stack([np.asarray(m, complex) for m in h.values()], axis=-1))
    return keys, blocks


def run(emul, h, k):
    keys, blocks = pack(h)
    n, nR = blocks.shape[0], blocks.shape[2]
    kp = np.array(k, float)
    ev = np.zeros(n)
    U = np.zeros((n, n), complex, order="F")
    emul.lqm_emul_eigh(n, nR, 2, blocks.ctypes.data_as(P), keys.ctypes.data_as(P), kp.ctypes.data_as(P), 1,
                       ev.ctypes.data_as(P), U.ctypes.data_as(P), None, None)
    return ev, U


def models():
    out = [("honeycomb144", M.honeycomb_disorder()[1])]
    out += M.batch_models()
    out.append(("tbg_n2", M.graphene(L.honeycomb_twisted(2), tz=0.32)))
    out.append(("single", {(0, 0): np.array([[0.7]], complex), (1, 0): np.array([[0.3]], complex),
                           (-1, 0): np.array([[0.3]], complex)}))
    return out


@pytest.mark.parametrize("name,h", models(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_eigh_matches_oracle(emul, name, h):
    for k in [(0.0, 0.0), (1 / 3, -1 / 3), (0.123, 0.77)]:
        ev, U = run(emul, h, k)
        Hk = K.fouriersum(h, k)
        ref = K.eigh_upper(Hk, vectors=False)
        n = len(ev)
        scale = max(ref[-1] - ref[0], 1.0)
        assert np.max(np.abs(ev - ref)) / scale <= 1e-12
        assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12
        assert np.max(np.abs(Hk @ U - U * ev)) / scale <= 1e-12


@pytest.mark.parametrize("nb,tile_min", [(32, 16), (5, 8), (8, 1 << 30)])
@pytest.mark.parametrize("name,h", models(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_blocked_eigh_matches_oracle(emul, name, h, nb, tile_min):
    """The large-n path (panel reduction, tiled merge updates, compact-WY back-transformation)."""
    keys, blocks = pack(h)
    n, nR = blocks.shape[0], blocks.shape[2]
    for k in [(0.0, 0.0), (0.123, 0.77)]:
        kp = np.array(k, float)
        ev = np.zeros(n)
        ev_only = np.zeros(n)
        U = np.zeros((n, n), complex, order="F")
        emul.lqm_emul_eigh_blocked(n, nR, 2, blocks.ctypes.data_as(P), keys.ctypes.data_as(P),
                                   kp.ctypes.data_as(P), nb, tile_min, 1, ev.ctypes.data_as(P), U.ctypes.data_as(P))
        emul.lqm_emul_eigh_blocked(n, nR, 2, blocks.ctypes.data_as(P), keys.ctypes.data_as(P),
                                   kp.ctypes.data_as(P), nb, tile_min, 0, ev_only.ctypes.data_as(P), None)
        Hk = K.fouriersum(h, k)
        ref = K.eigh_upper(Hk, vectors=False)
        scale = max(ref[-1] - ref[0], 1.0)
        assert np.max(np.abs(ev - ref)) / scale <= 1e-12
        assert np.max(np.abs(ev_only - ref)) / scale <= 1e-12
        assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12
        assert np.max(np.abs(Hk @ U - U * ev)) / scale <= 1e-12


@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 33, 64, 100])
def test_emulated_tridiagonal_dc(emul, n):
    rng = np.random.default_rng(n)
    for kind in ("random", "degenerate", "glued"):
        if kind == "random":
            d, e = rng.normal(size=n), rng.normal(size=max(n - 1, 0))
        elif kind == "degenerate":
            d = np.repeat(rng.normal(size=(n + 1) // 2), 2)[:n]
            e = np.zeros(max(n - 1, 0))
        else:
            d = np.abs(np.arange(n) - n // 2).astype(float)
            e = np.full(max(n - 1, 0), 1e-9)
        ev = np.zeros(n)
        Z = np.zeros((n, n), order="F")
        emul.lqm_emul_tridiag(n, d.ctypes.data_as(P), e.ctypes.data_as(P), ev.ctypes.data_as(P),
                              Z.ctypes.data_as(P), 1)
        ev_only = np.zeros(n)
        emul.lqm_emul_tridiag(n, d.ctypes.data_as(P), e.ctypes.data_as(P), ev_only.ctypes.data_as(P),
                              Z.ctypes.data_as(P), 0)
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        scale = max(np.max(np.abs(d)), 1.0)
        assert np.max(np.abs(ev - np.linalg.eigvalsh(T))) <= 1e-13 * scale
        assert np.max(np.abs(ev_only - np.linalg.eigvalsh(T))) <= 1e-13 * scale  # eigenvalue-only merges
        assert np.all(np.diff(ev) >= 0)
        assert np.max(np.abs(Z.T @ Z - np.eye(n))) <= 1e-13
        assert np.max(np.abs(T @ Z - Z * ev)) <= 1e-13 * scale


@pytest.mark.parametrize("n", [1, 5, 37, 96, 130])
def test_emulated_rho_from_U(emul, n):
    """rho = U f U^H for a unitary U, through both forms: the direct sum (more exact
    zeros than ones among f) and the complement I - U (1 - f) U^H (more exact ones)."""
    rng = np.random.default_rng(n)
    U, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    U = np.asfortranarray(U)
    for zeros, ones in ((slice(None, None, 3), slice(1, None, 5)), (slice(1, None, 5), slice(None, None, 3))):
        f = rng.random(n)
        f[zeros] = 0.0
        f[ones] = 1.0
        out = np.zeros((n, n), complex, order="F")
        emul.lqm_emul_rho(n, U.ctypes.data_as(P), f.ctypes.data_as(P), out.ctypes.data_as(P))
        assert np.max(np.abs(out - (U * f) @ U.conj().T)) < 1e-13 * max(n, 1)
        off = ~np.eye(n, dtype=bool)
        assert np.all(out[off] == out.conj().T[off])  # the lower triangle mirrors the upper exactly


@pytest.mark.parametrize("name,h", models()[1:4], ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_backtransform_column_range(emul, name, h):
    """The rho-only path transforms only a contiguous range of eigenvector columns: those
    columns come out bit-identical to the full back-transformation's."""
    keys, blocks = pack(h)
    n, nR = blocks.shape[0], blocks.shape[2]
    kp = np.array((0.123, 0.77), float)
    ev, Ufull = run(emul, h, (0.123, 0.77))
    for cb, ce in ((0, n // 2), (n // 3, n), (1, n - 1)):
        ev2 = np.zeros(n)
        U = np.zeros((n, n), complex, order="F")
        emul.lqm_emul_eigh_cols(n, nR, 2, blocks.ctypes.data_as(P), keys.ctypes.data_as(P), kp.ctypes.data_as(P),
                                cb, ce, ev2.ctypes.data_as(P), U.ctypes.data_as(P))
        assert np.array_equal(ev2, ev)
        assert np.array_equal(U[:, cb:ce], Ufull[:, cb:ce])


def _stress_tridiagonals():
    """Standard hard cases for divide and conquer: Wilkinson W+ (eigenvalue pairs
    split near machine precision), glued Wilkinson blocks (clusters of up to five),
    Clement (integer spectrum +-(n-1), +-(n-3), ...), the discrete Laplacian, graded
    entries, zero / constant / decoupled matrices and extreme scales."""
    out = []
    for m in (21, 97):
        k = (m - 1) // 2
        out.append((f"wilkinson{m}", np.abs(np.arange(-k, k + 1)).astype(float), np.ones(m - 1)))
    for delta in (1e-14, 1e-8):
        d = np.tile(np.abs(np.arange(-10, 11)).astype(float), 5)
        e = np.ones(len(d) - 1)
        e[20::21] = delta
        out.append((f"glued_wilkinson21x5_{delta:g}", d, e))
    for n in (10, 96):
        i = np.arange(1, n)
        out.append((f"clement{n}", np.zeros(n), np.sqrt(i * (n - i))))
    rng = np.random.default_rng(5)
    n = 96
    out += [("laplace96", np.full(n, 2.0), np.full(n - 1, -1.0)),
            ("graded96", 10.0 ** (-0.3 * np.arange(n)), 10.0 ** (-0.3 * np.arange(n - 1) - 0.15)),
            ("zero96", np.zeros(n), np.zeros(n - 1)),
            ("const96", np.full(n, 3.0), np.zeros(n - 1)),
            ("tiny_coupling96", rng.normal(size=n), np.full(n - 1, 1e-300)),
            ("scale1e150", rng.normal(size=n) * 1e150, rng.normal(size=n - 1) * 1e150),
            ("scale1e-150", rng.normal(size=n) * 1e-150, rng.normal(size=n - 1) * 1e-150)]
    return out


@pytest.mark.parametrize("name,d,e", _stress_tridiagonals(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_dc_stress_matrices(emul, name, d, e):
    n = len(d)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    ref = np.linalg.eigvalsh(T)
    scale = max(np.max(np.abs(ref)), np.finfo(float).tiny)
    for vec in (1, 0):
        ev = np.zeros(n)
        Z = np.zeros((n, n), order="F")
        emul.lqm_emul_tridiag(n, np.ascontiguousarray(d).ctypes.data_as(P), np.ascontiguousarray(e).ctypes.data_as(P),
                              ev.ctypes.data_as(P), Z.ctypes.data_as(P), vec)
        assert np.all(np.isfinite(ev)) and np.all(np.diff(ev) >= 0)
        assert np.max(np.abs(ev - ref)) <= 1e-13 * scale
        if vec:
            assert np.max(np.abs(Z.T @ Z - np.eye(n))) <= 1e-13
            assert np.max(np.abs(T @ Z - Z * ev)) <= 1e-13 * scale


def _hard_hermitian():
    rng = np.random.default_rng(9)

    def unitary(n):
        return np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))[0]

    def herm(n):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        return (A + A.conj().T) / 2

    out = []
    for n in (8, 96):
        e = rng.normal(size=n - 1) * np.exp(1j * rng.uniform(0, 2 * np.pi, n - 1))
        Q = unitary(n)
        dv = np.repeat(rng.normal(size=(n + 3) // 4), 4)[:n]
        Q2 = unitary(n)
        dp = np.sort(rng.normal(size=n))
        dp[1::2] = dp[0::2][:len(dp[1::2])] + 1e-13
        Mz = herm(n)
        Mz[:, n // 2] = 0
        Mz[n // 2, :] = 0
        out += [(f"diagonal{n}", np.diag(rng.normal(size=n)).astype(complex)),
                (f"tridiagonal_complex{n}", np.diag(rng.normal(size=n)) + np.diag(e, -1) + np.diag(e.conj(), 1)),
                (f"fourfold_degenerate{n}", Q @ np.diag(dv) @ Q.conj().T),
                (f"pairs_split_1e-13_{n}", Q2 @ np.diag(dp) @ Q2.conj().T),
                (f"zero{n}", np.zeros((n, n), complex)),
                (f"identity{n}", np.eye(n, dtype=complex)),
                (f"scale1e150_{n}", herm(n) * 1e150),
                (f"scale1e-150_{n}", herm(n) * 1e-150),
                (f"zero_row_and_column{n}", Mz),
                (f"rank_one{n}", 3.0 * np.outer(Q[:, 0], Q[:, 0].conj()))]
    return out


@pytest.mark.parametrize("name,Hk", _hard_hermitian(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_eigh_hard_hermitian(emul, name, Hk):
    """The whole one-CTA path (Householder, divide and conquer, back-transformation)
    on inputs that exercise its special cases: zero reflectors, deflation of whole
    clusters, near-degenerate pairs, extreme scales."""
    ev, U = run(emul, {(0, 0): Hk}, (0.0, 0.0))
    n = Hk.shape[0]
    ref = K.eigh_upper(Hk, vectors=False)
    scale = max(np.max(np.abs(ref)), np.finfo(float).tiny)
    assert np.all(np.isfinite(U))
    assert np.max(np.abs(ev - ref)) <= 1e-12 * scale
    assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12
    assert np.max(np.abs(Hk @ U - U * ev)) <= 1e-12 * scale


@pytest.mark.parametrize("name,Hk", _hard_hermitian(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_blocked_eigh_hard_hermitian(emul, name, Hk):
    """The same hard inputs through the large-n path's code (panel reduction with
    panels of 8, tiled merge updates from 8 rows, compact-WY back-transformation)."""
    keys, blocks = pack({(0, 0): Hk})
    n = Hk.shape[0]
    kp = np.zeros(2)
    ev = np.zeros(n)
    U = np.zeros((n, n), complex, order="F")
    emul.lqm_emul_eigh_blocked(n, 1, 2, blocks.ctypes.data_as(P), keys.ctypes.data_as(P), kp.ctypes.data_as(P),
                               8, 8, 1, ev.ctypes.data_as(P), U.ctypes.data_as(P))
    ref = K.eigh_upper(Hk, vectors=False)
    scale = max(np.max(np.abs(ref)), np.finfo(float).tiny)
    assert np.all(np.isfinite(U))
    assert np.max(np.abs(ev - ref)) <= 1e-12 * scale
    assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12
    assert np.max(np.abs(Hk @ U - U * ev)) <= 1e-12 * scale


def _run_two_stage(emul, h, k, b, want_vectors=True):
    keys, blocks = pack(h)
    n, nR = blocks.shape[0], blocks.shape[2]
    kp = np.array(k, float)
    ev = np.zeros(n)
    U = np.zeros((n, n), complex, order="F")
    tri = np.zeros(2 * n + 1)
    emul.lqm_emul_eigh_twostage(n, nR, 2, blocks.ctypes.data_as(P), keys.ctypes.data_as(P), kp.ctypes.data_as(P),
                                b, 1 if want_vectors else 0, ev.ctypes.data_as(P),
                                U.ctypes.data_as(P) if want_vectors else None, tri.ctypes.data_as(P))
    return ev, U, tri


@pytest.mark.parametrize("b", [4, 16, -4, -16])
@pytest.mark.parametrize("name,h", models(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_two_stage_eigh_matches_oracle(emul, name, h, b):
    """The two-stage reduction (panel QRs below a band of half-bandwidth |b| with the
    GEMM-form trailing update, the bulge chase to a real tridiagonal), divide and
    conquer, and the two-level back-transformation U = Q1 Q2 Z (b < 0: Q2 applied in
    the grouped order of the device kernel)."""
    for k in [(0.0, 0.0), (0.123, 0.77)]:
        ev, U, tri = _run_two_stage(emul, h, k, b)
        ev_only, _, _ = _run_two_stage(emul, h, k, b, want_vectors=False)
        n = len(ev)
        Hk = K.fouriersum(h, k)
        ref = K.eigh_upper(Hk, vectors=False)
        scale = max(ref[-1] - ref[0], 1.0)
        assert tri[2 * n] == 0.0  # nothing left outside the tridiagonal, subdiagonal real
        assert np.max(np.abs(ev - ref)) / scale <= 1e-12
        assert np.max(np.abs(ev_only - ref)) / scale <= 1e-12
        assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12
        assert np.max(np.abs(Hk @ U - U * ev)) / scale <= 1e-12


@pytest.mark.parametrize("name,Hk", _hard_hermitian(), ids=lambda x: x if isinstance(x, str) else "")
def test_emulated_two_stage_hard_hermitian(emul, name, Hk):
    """The hard inputs through the two-stage path (half-bandwidth 4: many panels and
    bulges on n = 8 and 96; 16 on n = 96)."""
    n = Hk.shape[0]
    ref = K.eigh_upper(Hk, vectors=False)
    scale = max(np.max(np.abs(ref)), np.finfo(float).tiny)
    for b in (4, 16, -16):
        ev, U, _ = _run_two_stage(emul, {(0, 0): Hk}, (0.0, 0.0), b)
        assert np.all(np.isfinite(U)), b
        assert np.max(np.abs(ev - ref)) <= 1e-12 * scale, b
        assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12, b
        assert np.max(np.abs(Hk @ U - U * ev)) <= 1e-12 * scale, b


@pytest.mark.parametrize("n", [3, 17, 18, 31, 33, 47, 65])
def test_emulated_two_stage_edge_orders(emul, n):
    """Orders around the half-bandwidth and its multiples (a last panel of 1 or b - 1
    rows, tasks cut at the matrix edge), dense random Hermitian H, both Q2 orders."""
    rng = np.random.default_rng(100 + n)
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    Hk = (A + A.conj().T) / 2
    ref = K.eigh_upper(Hk, vectors=False)
    scale = max(ref[-1] - ref[0], 1.0)
    for b in (4, 16, -4, -16):
        ev, U, tri = _run_two_stage(emul, {(0, 0): Hk}, (0.0, 0.0), b)
        assert tri[2 * n] == 0.0, b
        assert np.max(np.abs(ev - ref)) / scale <= 1e-12, b
        assert np.max(np.abs(U.conj().T @ U - np.eye(n))) <= 1e-12, b
        assert np.max(np.abs(Hk @ U - U * ev)) / scale <= 1e-12, b


@pytest.mark.parametrize("b,n", [(4, 61), (16, 200), (16, 131)])
def test_emulated_chase_concurrent_sweeps_match_sequential(emul, b, n):
    """The device chase runs successive sweeps concurrently, task t of sweep s waiting
    for task t + 2 of sweep s - 1.  Here the sweeps run on host threads with that
    protocol (acquire / release on the progress words, random pauses to vary the
    interleaving): the band, the reflectors and the taus must equal the sequential
    chase's bit for bit, for several schedules and worker counts."""
    rng = np.random.default_rng(n + b)
    ldb = 2 * b
    band = np.zeros((ldb, n), complex, order="F")  # element (i, j) at [i - j, j]
    for o in range(b + 1):
        band[o, : n - o] = rng.normal(size=n - o) + (1j * rng.normal(size=n - o) if o > 0 else 0.0)
    for workers, seed in ((8, 1), (8, 2), (3, 3), (13, 4)):
        assert emul.lqm_emul_chase_schedules(n, b, band.ctypes.data_as(P), workers, seed) == 1, (workers, seed)
