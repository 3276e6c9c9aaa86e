"""ctypes binding of the oracle's C++/OpenMP k-loop (cpu_kspace.cpp): the density
matrix and bands of LatticeQM.jl's `:multithreaded` path (per k: H(k), LAPACK
zheevr, rho_k = U f U^H, Fourier fold), on all host cores with one BLAS thread
per worker thread.  Test infrastructure: the checker and bench.py's CPU baseline."""
import ctypes
import os

import numpy as np

from oracle import build_cpu

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_cpu.LIB if os.path.exists(build_cpu.LIB) else build_cpu.build()
        _lib = ctypes.CDLL(path)
        P, I64, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        _lib.lqm_cpu_densitymatrix.argtypes = [I64, I64, ctypes.c_int32, P, P, I64, P, P, D, D, I64, P, P, P, P,
                                               ctypes.c_int]
        _lib.lqm_cpu_bandmatrix.argtypes = [I64, I64, ctypes.c_int32, P, P, I64, P, P, ctypes.c_int]
    return _lib


def _pack(h):
    keys = list(h.keys())
    n = np.asarray(h[keys[0]]).shape[0]
    K = np.ascontiguousarray(np.array(keys, dtype=np.int64))          # nR x d == d x nR column-major
    B = np.empty((len(keys), n, n), dtype=np.complex128)               # per key, column-major n x n
    for r, R in enumerate(keys):
        B[r] = np.asarray(h[R], dtype=np.complex128).T
    return n, len(keys), K.shape[1], K, B


def densitymatrix(h, ks, w, mu, T, Lkeys, nthreads=0, packed=None, want_bands=False):
    """rho (dict L -> n x n), eband[, bands n x nk] with the C++ k-loop."""
    n, nR, d, K, B = packed or _pack(h)
    ks = np.ascontiguousarray(np.asarray(ks, dtype=np.float64).T)      # nk x d == d x nk column-major
    nk = ks.shape[0]
    wv = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
    Lk = np.ascontiguousarray(np.array(Lkeys, dtype=np.int64))
    rho = np.zeros((len(Lkeys), n, n), dtype=np.complex128)
    eb = ctypes.c_double()
    bands = np.zeros((nk, n)) if want_bands else None
    st = lib().lqm_cpu_densitymatrix(n, nR, d, K.ctypes.data, B.ctypes.data, nk, ks.ctypes.data,
                                     None if wv is None else wv.ctypes.data, float(mu), float(T), len(Lkeys),
                                     Lk.ctypes.data, rho.ctypes.data, ctypes.byref(eb),
                                     None if bands is None else bands.ctypes.data, int(nthreads))
    if st != 0:
        raise RuntimeError(f"zheevr info {st}")
    out = {tuple(L): rho[i].T.copy() for i, L in enumerate(Lkeys)}
    if want_bands:
        return out, eb.value, bands.T.copy()
    return out, eb.value


def bandmatrix(h, ks, nthreads=0, packed=None):
    n, nR, d, K, B = packed or _pack(h)
    ks = np.ascontiguousarray(np.asarray(ks, dtype=np.float64).T)
    nk = ks.shape[0]
    bands = np.zeros((nk, n))
    st = lib().lqm_cpu_bandmatrix(n, nR, d, K.ctypes.data, B.ctypes.data, nk, ks.ctypes.data, bands.ctypes.data,
                                  int(nthreads))
    if st != 0:
        raise RuntimeError(f"zheevr info {st}")
    return bands.T.copy()


def max_threads():
    return int(lib().lqm_cpu_max_threads())
