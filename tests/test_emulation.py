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
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", inc, src, "-o", str(out)], check=True)
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
