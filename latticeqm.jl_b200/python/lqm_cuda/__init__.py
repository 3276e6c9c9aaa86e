"""ctypes mirror of LatticeQM's k-space routines on the ``multimode=:cuda`` path.

This is the Python twin of the Julia glue (``latticeqm.jl_b200/julia/LatticeQMCUDA.jl``):
the same names, argument meanings and layouts as the reference routines, each
one a thin call into ``libkspace.so`` (include/kspace.h).  There is no CPU
fallback: importing this module without the built library, or calling it
without a CUDA device, raises.

Hops are dicts ``{R (tuple of ints): ndarray (n, n) complex128}`` in the
reference's key order (the Bloch-sum order).  k-points are fractional, shape
(d, nk).  Arrays follow Julia's column-major layout at the C boundary.

Reference (LatticeQM.jl):
  bandmatrix / getbands        src/modules/Spectrum/bands.jl:164-204,264-267
  getdensitymatrix!            src/modules/Operators/densitymatrix.jl:17-49
  chemicalpotential            src/modules/Spectrum/chemicalpotential.jl:6-66
  getdos                       src/modules/Spectrum/dos.jl:127-223
  solvehartreefock             src/modules/Meanfield/selfconsistent.jl:19-104
"""
import ctypes
import os
import warnings
from collections import namedtuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get(
    "LQM_KSPACE_LIB", os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libkspace.so")))

LQM_OK = 0
LQM_ETIMEOUT = -4
STATUS_NAMES = {-1: "LQM_EINVAL", -2: "LQM_ECUDA", -3: "LQM_ENOMEM", -4: "LQM_ETIMEOUT",
                -5: "LQM_ENOCONV", -6: "LQM_EDEVICE"}

EXPORTS = [
    "lqm_ctx_create", "lqm_ctx_destroy", "lqm_last_error", "lqm_ctx_set_timeout", "lqm_ctx_set_blocked_min_n",
    "lqm_ctx_set_two_stage", "lqm_ctx_set_device_wait_limit",
    "lqm_ctx_last_kernel_ms", "lqm_hops_upload_dense", "lqm_hops_upload_csc", "lqm_hops_free",
    "lqm_hops_dims", "lqm_bloch", "lqm_bloch_dev", "lqm_bandmatrix", "lqm_bandmatrix_dev",
    "lqm_densitymatrix", "lqm_densitymatrix_dev", "lqm_chemicalpotential",
    "lqm_chemicalpotential_bands_dev", "lqm_dos", "lqm_dos_bands_dev", "lqm_scf_hf",
    "lqm_ctx_reset_stats", "lqm_ctx_stats", "lqm_bands_dos_rho", "lqm_bands_dos_rho_dev",
    "lqm_ctx_phase_cycles", "lqm_bandmatrix_noalloc", "lqm_densitymatrix_vjp", "lqm_bands_vjp",
    "lqm_bandmatrix_obs", "lqm_ctx_set_scf_acceleration", "lqm_density", "lqm_ldos",
    "lqm_berry", "lqm_opticalconductivity", "lqm_bandmatrix_partial", "lqm_densitymatrix_partial",
    "lqm_commutator_norm", "lqm_ctx_set_scf_residual", "lqm_ctx_set_scf_terms", "lqm_ctx_set_scf_exchange",
    "lqm_ctx_scf_exchange_energy", "lqm_hartreefock_eval", "lqm_bdg_densitymatrix", "lqm_bdg_filling",
    "lqm_bdg_chemicalpotential", "lqm_scf_hf_bdg", "lqm_berry_flux", "lqm_berry_path", "lqm_fermisurface",
    "lqm_wilson", "lqm_wilson_wannier", "lqm_ctx_set_eigh_threads", "lqm_autotune_eigh", "lqm_ctx_kernel_stats",
    "lqm_comm_unique_id", "lqm_ctx_set_comm", "lqm_ctx_comm", "lqm_shard_range", "lqm_scf_hf_gradient",
    "lqm_bands_dos_rho_multi_dev",
]


class LQMError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


if not os.path.exists(LIB_PATH):
    raise ImportError(f"libkspace.so not built at {LIB_PATH}; run latticeqm.jl_b200/build.py")

_lib = ctypes.CDLL(LIB_PATH)
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
LOG_CB = ctypes.CFUNCTYPE(ctypes.c_int, _I64, _D, _D, _D, _D, _D, _D, _D, _P)

_SIG = {
    "lqm_ctx_create": [ctypes.c_int, ctypes.POINTER(_P)],
    "lqm_ctx_destroy": [_P],
    "lqm_ctx_set_timeout": [_P, _D],
    "lqm_ctx_set_blocked_min_n": [_P, _I64],
    "lqm_ctx_set_two_stage": [_P, ctypes.c_int],
    "lqm_ctx_set_device_wait_limit": [_P, _I64],
    "lqm_ctx_kernel_stats": [_P, ctypes.c_int, ctypes.POINTER(_D), ctypes.POINTER(_I64), ctypes.POINTER(_D)],
    "lqm_comm_unique_id": [_P],
    "lqm_ctx_set_comm": [_P, ctypes.c_int, ctypes.c_int, _P],
    "lqm_ctx_comm": [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
    "lqm_shard_range": [_I64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
    "lqm_scf_hf_gradient": [_P, _P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, _P, _D, _D, _I64, _P, _P, _P],
    "lqm_bands_dos_rho_multi_dev": [_P, ctypes.c_int, _P, _I64, _P, _P, _D, _D, _P, _P, _P, _P, _I64, _P, _D, _P, _P],
    "lqm_ctx_last_kernel_ms": [_P, ctypes.POINTER(_D)],
    "lqm_hops_upload_dense": [_P, _I64, _I64, ctypes.c_int32, _P, _P, ctypes.POINTER(_P)],
    "lqm_hops_upload_csc": [_P, _I64, _I64, ctypes.c_int32, _P, _P, _P, _P, _P, ctypes.POINTER(_P)],
    "lqm_hops_free": [_P, _P],
    "lqm_hops_dims": [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(ctypes.c_int32)],
    "lqm_bloch": [_P, _P, _I64, _P, _P],
    "lqm_bloch_dev": [_P, _P, _I64, _P, _P],
    "lqm_bandmatrix": [_P, _P, _I64, _P, ctypes.c_int, ctypes.c_int, _P, _P],
    "lqm_bandmatrix_dev": [_P, _P, _I64, _P, ctypes.c_int, ctypes.c_int, _P, _P],
    "lqm_densitymatrix": [_P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, ctypes.POINTER(_D), ctypes.c_int],
    "lqm_densitymatrix_dev": [_P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, ctypes.POINTER(_D),
                              ctypes.c_int],
    "lqm_chemicalpotential": [_P, _P, _I64, _P, _P, _D, _D, ctypes.POINTER(_D)],
    "lqm_chemicalpotential_bands_dev": [_P, _I64, _I64, _P, _P, _D, _D, ctypes.POINTER(_D)],
    "lqm_dos": [_P, _P, _I64, _P, _P, _I64, _P, _D, _P],
    "lqm_dos_bands_dev": [_P, _I64, _I64, _P, _P, _I64, _P, _D, _P],
    "lqm_scf_hf": [_P, _P, _P, _I64, _P, _P, _D, _D, _D, _D, _I64, _I64, _P, _P, LOG_CB, _P, _P],
    "lqm_ctx_reset_stats": [_P, ctypes.c_int],
    "lqm_ctx_phase_cycles": [_P, ctypes.POINTER(_D)],
    "lqm_bandmatrix_noalloc": [_P, _I64, _I64, ctypes.c_int32, _P, _P, _I64, _P, _P, _P],
    "lqm_ctx_stats": [_P, ctypes.POINTER(_D), ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
    "lqm_densitymatrix_vjp": [_P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, _P],
    "lqm_bands_vjp": [_P, _P, _I64, _P, _P, _P],
    "lqm_bandmatrix_obs": [_P, _P, _I64, _P, _I64, _P, _P, _P],
    "lqm_ctx_set_scf_acceleration": [_P, ctypes.c_int],
    "lqm_density": [_P, _P, _I64, _P, _D, _P],
    "lqm_ldos": [_P, _P, _I64, _P, _I64, _P, _D, _P],
    "lqm_berry": [_P, _P, _I64, _I64, _I64, _P, _P],
    "lqm_berry_flux": [_P, _P, _I64, _I64, _I64, _P, _P, _P],
    "lqm_berry_path": [_P, _P, _I64, _P, _P],
    "lqm_wilson": [_P, _P, _I64, _I64, _I64, _P, ctypes.c_int, _P, _P],
    "lqm_wilson_wannier": [_P, _P, _I64, _I64, _I64, _P, _P, _P],
    "lqm_ctx_set_eigh_threads": [_P, _I64, ctypes.c_int],
    "lqm_autotune_eigh": [_P, _P, _I64, _P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_D), _I64,
                          _P, _P, ctypes.POINTER(_I64)],
    "lqm_fermisurface": [_P, _P, _I64, _P, _I64, _P, _D, _P, _P, ctypes.POINTER(_D)],
    "lqm_opticalconductivity": [_P, _P, _P, _P, _I64, _P, _I64, _P, _D, _D, _D, _P],
    "lqm_commutator_norm": [_P, _P, _P, _I64, _P, _P, ctypes.POINTER(_D)],
    "lqm_ctx_set_scf_residual": [_P, ctypes.c_int],
    "lqm_ctx_set_scf_terms": [_P, ctypes.c_int, ctypes.c_int],
    "lqm_ctx_set_scf_exchange": [_P, _I64, _I64, ctypes.c_int32, _P, _P, _I64, _P, _P],
    "lqm_ctx_scf_exchange_energy": [_P, ctypes.POINTER(_D)],
    "lqm_hartreefock_eval": [_P, _P, _P, _I64, _P, _P, _I64, _P, _P, _P],
    "lqm_bdg_densitymatrix": [_P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, ctypes.POINTER(_D)],
    "lqm_bdg_filling": [_P, _P, _I64, _P, _P, _D, _D, ctypes.POINTER(_D)],
    "lqm_bdg_chemicalpotential": [_P, _P, _I64, _P, _P, _D, _D, _D, _D, ctypes.POINTER(_D)],
    "lqm_scf_hf_bdg": [_P, _P, _P, _I64, _P, _D, _D, _D, _D, _I64, _I64, _P, _P, LOG_CB, _P, _P],
    "lqm_bandmatrix_partial": [_P, _P, _I64, _P, _I64, _D, ctypes.c_int, ctypes.c_int, _P, _P],
    "lqm_densitymatrix_partial": [_P, _P, _I64, _P, _P, _D, _D, _I64, _D, ctypes.c_int, _I64, _P, _P,
                                  ctypes.POINTER(_D)],
    "lqm_bands_dos_rho": [_P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, ctypes.POINTER(_D), _I64, _P, _D, _P,
                          _P, ctypes.c_int],
    "lqm_bands_dos_rho_dev": [_P, _P, _I64, _P, _P, _D, _D, _I64, _P, _P, ctypes.POINTER(_D), _I64, _P, _D,
                              _P, _P, ctypes.c_int],
}
for _name, _args in _SIG.items():
    _f = getattr(_lib, _name)
    _f.argtypes = _args
    _f.restype = ctypes.c_int
_lib.lqm_last_error.argtypes = [_P]
_lib.lqm_last_error.restype = ctypes.c_char_p


def lib():
    return _lib


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # device tensor (torch) for the _dev entry points
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(_P)


class Context:
    """One CUDA device + stream (``lqm_ctx``)."""

    def __init__(self, device=0, timeout=None):
        h = _P()
        st = _lib.lqm_ctx_create(int(device), ctypes.byref(h))
        if st != LQM_OK:
            raise LQMError(st, f"cannot create a context on CUDA device {device}")
        self._h = h
        self.device = int(device)
        if timeout is not None:
            self.check(_lib.lqm_ctx_set_timeout(self._h, float(timeout)))

    @property
    def handle(self):
        return self._h

    def check(self, st):
        if st != LQM_OK:
            raise LQMError(st, (_lib.lqm_last_error(self._h) or b"").decode())

    def set_blocked_min_n(self, n_min):
        """Orders n >= n_min use the batched blocked eigensolver (0: only where the
        one-CTA-per-k kernel does not fit)."""
        self.check(_lib.lqm_ctx_set_blocked_min_n(self._h, int(n_min)))

    def set_two_stage(self, mode):
        """Reduction of the blocked eigensolver: 1 two-stage (dense -> band -> tridiagonal),
        0 one-stage panels, -1 (default): two-stage on the blocked path for passes that
        return no eigenvectors."""
        self.check(_lib.lqm_ctx_set_two_stage(self._h, int(mode)))

    def set_device_wait_limit(self, polls):
        """Polls before a device-side wait of the bulge chase gives up (0: the default)."""
        self.check(_lib.lqm_ctx_set_device_wait_limit(self._h, int(polls)))

    def set_eigh_threads(self, n, nt):
        """Block size of the one-CTA eigensolver for order n (0: the built-in rule)."""
        self.check(_lib.lqm_ctx_set_eigh_threads(self._h, int(n), int(nt)))

    def last_kernel_ms(self):
        v = _D()
        self.check(_lib.lqm_ctx_last_kernel_ms(self._h, ctypes.byref(v)))
        return v.value

    def reset_stats(self, timing=True, phases=False):
        """Zero the statistics; ``timing`` records CUDA-event times of the eigensolver
        launches, ``phases`` also its per-phase cycle counters (see ``phase_cycles``)."""
        mode = 2 if phases else int(bool(timing))
        self.check(_lib.lqm_ctx_reset_stats(self._h, mode))

    def stats(self):
        """(eigensolver device ms, eigensolver launches, all kernel launches) since reset."""
        ms, el, al = _D(), _I64(), _I64()
        self.check(_lib.lqm_ctx_stats(self._h, ctypes.byref(ms), ctypes.byref(el), ctypes.byref(al)))
        return ms.value, el.value, al.value

    def set_comm(self, nranks, rank, uid=None):
        """Join the k-point shards of `nranks` processes (one GPU each) as `rank`, with the
        communicator id from comm_unique_id() on rank 0 (bytes, shared by the caller);
        nranks = 1 without an id removes the communicator (with an id: a one-rank
        communicator, the sharded code path with copies for collectives)."""
        buf = None
        if nranks > 1 or uid is not None:
            if uid is None or len(uid) != COMM_ID_BYTES:
                raise ValueError(f"communicator id must be {COMM_ID_BYTES} bytes")
            buf = ctypes.create_string_buffer(bytes(uid), COMM_ID_BYTES)
        self.check(_lib.lqm_ctx_set_comm(self._h, int(nranks), int(rank), buf))

    def comm(self):
        """(nranks, rank) of the context's communicator ((1, 0) without one)."""
        nr, r = ctypes.c_int(), ctypes.c_int()
        self.check(_lib.lqm_ctx_comm(self._h, ctypes.byref(nr), ctypes.byref(r)))
        return nr.value, r.value

    def kernel_stats(self, kernel_class):
        """(device ms, launches, algorithmic amount) since reset for a kernel class:
        0 = eigensolver passes, 1 = the one-stage mat-vec kernel (bytes), 2 = the
        two-stage path's stage-2 back-transformation (flops)."""
        ms, nl, by = _D(), _I64(), _D()
        self.check(_lib.lqm_ctx_kernel_stats(self._h, int(kernel_class), ctypes.byref(ms), ctypes.byref(nl),
                                             ctypes.byref(by)))
        return ms.value, nl.value, by.value

    def phase_cycles(self):
        """Eigensolver SM cycles per stage: bloch, householder, d&c, back-transform, sync,
        then the d&c merge steps (zsort, deflate, secular, zhat, vectors, ranks, update, copy),
        then the householder steps (pass, mat-vec reduction, column); recorded after
        ``reset_stats(phases=True)``."""
        out = (_D * 16)()
        self.check(_lib.lqm_ctx_phase_cycles(self._h, out))
        return list(out)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lqm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


COMM_ID_BYTES = 128


def comm_unique_id():
    """A new communicator id (bytes) for Context.set_comm; made on one rank and shared."""
    buf = ctypes.create_string_buffer(COMM_ID_BYTES)
    st = _lib.lqm_comm_unique_id(buf)
    if st != LQM_OK:
        raise LQMError(st, "lqm_comm_unique_id failed (NCCL not loadable?)")
    return buf.raw


def shard_range(nk, nranks, rank):
    """[k0, k1) of the k list that `rank` of `nranks` processes (host only, no device)."""
    k0, k1 = _I64(), _I64()
    st = _lib.lqm_shard_range(int(nk), int(nranks), int(rank), ctypes.byref(k0), ctypes.byref(k1))
    if st != LQM_OK:
        raise LQMError(st, "invalid shard arguments")
    return k0.value, k1.value


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def pack_hops(h):
    """dict Hops -> (n, nR, d, keys d x nR int64 (F), blocks n x n x nR complex (F))."""
    keys = list(h.keys())
    mats = [np.asarray(h[R], dtype=np.complex128) for R in keys]
    n = mats[0].shape[0]
    d = len(keys[0])
    K = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    B = np.empty((n, n, len(keys)), dtype=np.complex128, order="F")  # one copy per block
    for r, m in enumerate(mats):
        B[:, :, r] = m
    return n, len(keys), d, K, B


def _is_sparse(m):
    return hasattr(m, "tocsc") and hasattr(m, "nnz")


def pack_hops_csc(h):
    """dict Hops of sparse (or dense) blocks -> (n, nR, d, keys d x nR int64 (F), per key
    the SparseMatrixCSC arrays as Julia holds them: 1-based int64 colptr and rowval,
    complex128 nzval)."""
    import scipy.sparse as sp
    keys = list(h.keys())
    d = len(keys[0])
    K = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    cols = []
    n = None
    for R in keys:
        m = h[R]
        c = m.tocsc() if _is_sparse(m) else sp.csc_matrix(np.asarray(m))
        n = c.shape[0]
        cols.append((np.ascontiguousarray(c.indptr, dtype=np.int64) + 1,
                     np.ascontiguousarray(c.indices, dtype=np.int64) + 1,
                     np.ascontiguousarray(c.data, dtype=np.complex128)))
    return n, len(keys), d, K, cols


class DeviceHops:
    """A Hops resident on the device (``lqm_hops``)."""

    def __init__(self, h, ctx=None):
        self.ctx = ctx or default_context()
        self.keys = [tuple(R) for R in h.keys()]
        out = _P()
        if any(_is_sparse(m) for m in h.values()):
            n, nR, d, K, cols = pack_hops_csc(h)
            self.n, self.nR, self.d = n, nR, d
            arr = ctypes.c_void_p * nR
            cp = arr(*[c.ctypes.data for c, _, _ in cols])
            rv = arr(*[r.ctypes.data for _, r, _ in cols])
            nz = arr(*[v.ctypes.data for _, _, v in cols])
            nnz = np.array([r.size for _, r, _ in cols], dtype=np.int64)
            self.ctx.check(_lib.lqm_hops_upload_csc(self.ctx.handle, n, nR, d, _ptr(K), ctypes.cast(cp, _P),
                                                    ctypes.cast(rv, _P), ctypes.cast(nz, _P), _ptr(nnz),
                                                    ctypes.byref(out)))
        else:
            n, nR, d, K, B = pack_hops(h)
            self.n, self.nR, self.d = n, nR, d
            self.ctx.check(_lib.lqm_hops_upload_dense(self.ctx.handle, n, nR, d, _ptr(K), _ptr(B),
                                                      ctypes.byref(out)))
        self._h = out

    @property
    def handle(self):
        return self._h

    def free(self):
        if getattr(self, "_h", None):
            st = _lib.lqm_hops_free(self.ctx.handle, self._h)
            if st == LQM_ETIMEOUT:  # device work still reads the blocks: the handle stays valid
                self.ctx.check(st)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _as_device_hops(H, ctx):
    return H if isinstance(H, DeviceHops) else DeviceHops(H, ctx)


def _hops_dims(H):
    """(n, d) of a dict Hops or a DeviceHops, without touching the device."""
    if isinstance(H, DeviceHops):
        return H.n, H.d
    R = next(iter(H))
    return np.asarray(H[R]).shape[0], len(R)


def _ks(ks, d=None):
    ks = np.asfortranarray(np.asarray(ks, dtype=np.float64))
    if ks.ndim == 1:
        ks = ks.reshape(-1, 1, order="F")
    if d is not None and ks.shape[0] != d:
        raise ValueError(f"k-points must have {d} rows, got {ks.shape[0]}")
    return ks


def _check_mode(multimode):
    if str(multimode).lstrip(":") != "cuda":
        raise ValueError(f"multimode={multimode!r}: this module implements only :cuda")


def bloch(H, ks, ctx=None):
    """H(k) for every column of ks: array (n, n, nk)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    nk = ks.shape[1]
    out = np.zeros((Hd.n, Hd.n, nk), dtype=np.complex128, order="F")
    ctx.check(_lib.lqm_bloch(ctx.handle, Hd.handle, nk, _ptr(ks), _ptr(out)))
    return out


def bandmatrix(H, ks, multimode="cuda", want_vectors=False, precision=0, ctx=None, format="dense",
               num_bands=None, sigma=1e-8, which="LM"):
    """``bandmatrix(H, ks)``: bands (n, nk) ascending per column; with
    ``want_vectors`` also U (n, n, nk) (columns = eigenvectors).  ``format="sparse"``
    with ``num_bands`` is the partial spectrum of ``bandmatrix_partial``."""
    _check_mode(multimode)
    if str(format).lstrip(":") == "sparse" and num_bands is not None:
        return bandmatrix_partial(H, ks, num_bands, sigma=sigma, which=which, want_vectors=want_vectors, ctx=ctx)
    n, d = _hops_dims(H)
    ks = _ks(ks, d)
    if ks.shape[1] == 0:  # an empty k-set: the reference's k-loop runs zero times (bands.jl:164-204)
        return np.zeros((n, 0), order="F"), (np.zeros((n, n, 0), dtype=np.complex128, order="F")
                                             if want_vectors else None)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    nk = ks.shape[1]
    bands = np.zeros((Hd.n, nk), order="F")
    U = np.zeros((Hd.n, Hd.n, nk), dtype=np.complex128, order="F") if want_vectors else None
    ctx.check(_lib.lqm_bandmatrix(ctx.handle, Hd.handle, nk, _ptr(ks), int(bool(want_vectors)),
                                  int(precision), _ptr(bands), _ptr(U)))
    return bands, U


BandData = namedtuple("BandData", ["bands", "obs", "path"])


def _projector_hops(op, n):
    """ExpvalMap operand (bands.jl:52-60) as Hops: a matrix -> {0: matrix}; a dict Hops as is."""
    if isinstance(op, dict):
        return op
    M = np.asarray(op, dtype=np.complex128)
    if M.shape != (n, n):
        raise ValueError(f"projector must be an {n} x {n} matrix or a Hops dict")
    return {(0, 0): M}


def bandmatrix_obs(H, ks, projectors, multimode="cuda", ctx=None):
    """``bandmatrix(H, ks, projectors...)``: bands (n, nk) and obs (n, nk, nproj) with
    obs[i, j, p] = Re <u_i(k_j)| P_p(k_j) |u_i(k_j)> (``lqm_bandmatrix_obs``)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    nk = ks.shape[1]
    Pd = [DeviceHops(_projector_hops(op, Hd.n), ctx) for op in projectors]
    arr = (_P * max(1, len(Pd)))(*[p.handle for p in Pd])
    bands = np.zeros((Hd.n, nk), order="F")
    obs = np.zeros((Hd.n, nk, len(Pd)), order="F")
    ctx.check(_lib.lqm_bandmatrix_obs(ctx.handle, Hd.handle, nk, _ptr(ks), len(Pd), arr, _ptr(bands),
                                      _ptr(obs) if Pd else None))
    return bands, obs


def getbands(H, ks, projectors=(), multimode="cuda", ctx=None):
    """``getbands(H, ks[, projectors])`` -> BandData(bands, obs, path)."""
    if projectors is None or (not isinstance(projectors, (list, tuple))):
        projectors = [] if projectors is None else [projectors]
    if len(projectors) == 0:
        bands, _ = bandmatrix(H, ks, multimode=multimode, ctx=ctx)
        return BandData(bands, np.zeros(bands.shape + (0,)), ks)
    bands, obs = bandmatrix_obs(H, ks, projectors, multimode=multimode, ctx=ctx)
    return BandData(bands, obs, ks)


_WHICH = {"LM": 0, "SR": 1, "LR": 2}


def _which(which):
    key = str(which).lstrip(":")
    if key not in _WHICH:
        raise ValueError(f"which={which!r}: use :LM, :SR or :LR")
    return _WHICH[key]


def bandmatrix_partial(H, ks, num_bands, sigma=1e-8, which="LM", want_vectors=False, ctx=None):
    """``bandmatrix(H, ks; format=:sparse, num_bands, sigma, which)``: per k the
    ``num_bands`` eigenvalues nearest ``sigma`` (:LM), smallest (:SR) or largest (:LR),
    ascending; bands (num_bands, nk) and optionally U (n, num_bands, nk)
    (``lqm_bandmatrix_partial``)."""
    n, d = _hops_dims(H)
    ks = _ks(ks, d)
    if ks.shape[1] == 0:
        return np.zeros((int(num_bands), 0), order="F"), (
            np.zeros((n, int(num_bands), 0), dtype=np.complex128, order="F") if want_vectors else None)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    nk = ks.shape[1]
    bands = np.zeros((int(num_bands), nk), order="F")
    U = np.zeros((Hd.n, int(num_bands), nk), dtype=np.complex128, order="F") if want_vectors else None
    ctx.check(_lib.lqm_bandmatrix_partial(ctx.handle, Hd.handle, nk, _ptr(ks), int(num_bands), float(sigma),
                                          _which(which), int(bool(want_vectors)), _ptr(bands), _ptr(U)))
    return bands, U


def getdensitymatrix(rhos, H, ks, kweights=None, mu=0.0, T=0.01, multimode="cuda", precision=0,
                     ctx=None, format="dense", num_bands=None, sigma=1e-8, which="LM"):
    """``getdensitymatrix!(ρs, H, ks[, kweights], μ; T[, format=:sparse, num_bands])``:
    overwrites every block of ``rhos`` (dict keyed like Hops; only its existing keys are
    computed) and returns the band energy sum_k w_k sum_n f eps.  With
    ``format="sparse"`` only the ``num_bands`` states selected as in
    ``bandmatrix_partial`` enter (``lqm_densitymatrix_partial``)."""
    _check_mode(multimode)
    n, d = _hops_dims(H)
    ks = _ks(ks, d)
    if ks.shape[1] == 0:  # an empty k-set: rho is zeroed and the k-sum is empty (densitymatrix.jl:17-49)
        for L in list(rhos.keys()):
            rhos[L] = np.zeros((n, n), dtype=np.complex128)
        return 0.0
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    nk = ks.shape[1]
    Lkeys = list(rhos.keys())
    nL = len(Lkeys)
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = np.zeros((Hd.n, Hd.n, nL), dtype=np.complex128, order="F")
    eb = _D()
    if str(format).lstrip(":") == "sparse":
        nbands = Hd.n if num_bands is None else int(num_bands)
        ctx.check(_lib.lqm_densitymatrix_partial(ctx.handle, Hd.handle, nk, _ptr(ks), _ptr(w), float(mu),
                                                 float(T), nbands, float(sigma), _which(which), nL, _ptr(Lk),
                                                 _ptr(out), ctypes.byref(eb)))
    else:
        ctx.check(_lib.lqm_densitymatrix(ctx.handle, Hd.handle, nk, _ptr(ks), _ptr(w), float(mu), float(T),
                                         nL, _ptr(Lk), _ptr(out), ctypes.byref(eb), int(precision)))
    for i, L in enumerate(Lkeys):
        rhos[L] = np.array(out[:, :, i])
    return eb.value


def densitymatrix_vjp(H, ks, Gbar, kweights=None, mu=0.0, T=0.01, ctx=None):
    """Reverse-mode derivative of ``getdensitymatrix!`` at fixed mu and T
    (``lqm_densitymatrix_vjp``).  ``Gbar``: dict L -> n x n cotangent dLoss/d rho_L.
    Returns dict R -> n x n (H's keys) with dLoss = Re sum_R <Hbar_R, dH_R> for
    Hermitian-consistent dH."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    Lkeys = list(Gbar.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    G = np.asfortranarray(np.stack([np.asarray(Gbar[L], dtype=np.complex128) for L in Lkeys], axis=-1))
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = np.zeros((Hd.n, Hd.n, Hd.nR), dtype=np.complex128, order="F")
    ctx.check(_lib.lqm_densitymatrix_vjp(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(w), float(mu),
                                         float(T), len(Lkeys), _ptr(Lk), _ptr(G), _ptr(out)))
    return {R: np.array(out[:, :, i]) for i, R in enumerate(Hd.keys)}


def bands_vjp(H, ks, eps_bar, ctx=None):
    """Reverse-mode derivative of ``bandmatrix``: eps_bar (n, nk) = dLoss/d bands ->
    dict R -> n x n with Hbar_R = sum_k e^{-i2pi k.R} U diag(eps_bar_k) U^H."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    eb = np.asfortranarray(np.asarray(eps_bar, dtype=np.float64))
    if eb.shape != (Hd.n, ks.shape[1]):
        raise ValueError("eps_bar must have shape (n, nk)")
    out = np.zeros((Hd.n, Hd.n, Hd.nR), dtype=np.complex128, order="F")
    ctx.check(_lib.lqm_bands_vjp(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(eb), _ptr(out)))
    return {R: np.array(out[:, :, i]) for i, R in enumerate(Hd.keys)}


def density(H, ks, mu=0.0, multimode="cuda", ctx=None):
    """``density(H, ks, μ)`` (Spectrum/dos.jl:20-52): per-orbital occupation of the
    states with eps <= mu, averaged over ks (``lqm_density``)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    out = np.zeros(Hd.n)
    ctx.check(_lib.lqm_density(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), float(mu), _ptr(out)))
    return out


def ldos(H, ks, frequencies, gamma=0.1, multimode="cuda", ctx=None):
    """``ldos(H, ks, frequencies; Γ)`` (Spectrum/dos.jl:56-98), with 1/π, averaged over
    the frequencies (``lqm_ldos``)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    om = np.ascontiguousarray(np.atleast_1d(frequencies), dtype=np.float64)
    out = np.zeros(Hd.n)
    ctx.check(_lib.lqm_ldos(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), len(om), _ptr(om), float(gamma),
                            _ptr(out)))
    return out


def berry(H, NX, NY=0, bands=(0,), multimode="cuda", ctx=None):
    """``berry(H, NX, NY, bandindices)`` (Spectrum/berry.jl:140-155) with 0-based band
    indices: returns (midkgrid (2, NX-1, NY-1), F (NX-1, NY-1)) like the reference."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    NY = NX if NY < 1 else NY
    b = np.ascontiguousarray(bands, dtype=np.int64)
    F = np.zeros((NX - 1, NY - 1), order="F")
    ctx.check(_lib.lqm_berry(ctx.handle, Hd.handle, int(NX), int(NY), len(b), _ptr(b), _ptr(F)))
    mx = np.linspace(0.5 / (NX - 1), 1 - 0.5 / (NX - 1), NX - 1)
    my = np.linspace(0.5 / (NY - 1), 1 - 0.5 / (NY - 1), NY - 1)
    mid = np.stack(np.meshgrid(mx, my, indexing="ij"))
    return mid, F


def opticalconductivity(frequencies, H, J1, J2, ks, mu=0.0, Gamma=0.025, T=0.1, multimode="cuda", ctx=None):
    """``opticalconductivity(frequencies, H, J1, J2, ks; μ, Γ, T)``
    (LinearResponse/opticalconductivity.jl:101-127): the Kubo current-current
    correlator chi(w) (complex, one per frequency; ``lqm_opticalconductivity``).
    J1, J2 are Hops of H's order (the current operators)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    J1d = _as_device_hops(J1, ctx)
    J2d = J1d if J2 is J1 else _as_device_hops(J2, ctx)  # one handle: the J2 = J1 shortcut
    om = np.ascontiguousarray(np.atleast_1d(frequencies), dtype=np.float64)
    out = np.zeros(len(om), dtype=np.complex128)
    ctx.check(_lib.lqm_opticalconductivity(ctx.handle, Hd.handle, J1d.handle, J2d.handle, ks.shape[1], _ptr(ks),
                                           len(om), _ptr(om), float(mu), float(Gamma), float(T), _ptr(out)))
    return out


def bdg_getdensitymatrix(rhos, H, ks, kweights=None, mu=0.0, T=0.01, ctx=None):
    """``getdensitymatrix!(ρ::BdGOperator, H::BdGOperator, ks[, kweights], μ; T)``
    (Superconductivity/green.jl:38-54) for a Nambu Hops ``H`` (order 2d): overwrites the
    blocks of ``rhos`` and returns ⟨H − μN⟩ (``lqm_bdg_densitymatrix``)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    Lkeys = list(rhos.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = np.zeros((Hd.n, Hd.n, len(Lkeys)), dtype=np.complex128, order="F")
    e = _D()
    ctx.check(_lib.lqm_bdg_densitymatrix(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(w), float(mu), float(T),
                                         len(Lkeys), _ptr(Lk), _ptr(out), ctypes.byref(e)))
    for i, L in enumerate(Lkeys):
        rhos[L] = np.array(out[:, :, i])
    return e.value


def bdg_filling(H, ks, mu=0.0, T=0.01, kweights=None, ctx=None):
    """``Spectrum.filling(H::BdGOperator, ks, μ; T)`` (Superconductivity/operators.jl:117-122)
    (``lqm_bdg_filling``)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = _D()
    ctx.check(_lib.lqm_bdg_filling(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(w), float(mu), float(T),
                                   ctypes.byref(out)))
    return out.value


def bdg_chemicalpotential(H, ks, filling, T=0.01, kweights=None, mu_lo=-100.0, mu_hi=100.0, ctx=None):
    """``Spectrum.chemicalpotential(H::BdGOperator, ks, target; T, μ_lo, μ_hi)``
    (Superconductivity/operators.jl:139-155) (``lqm_bdg_chemicalpotential``)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = _D()
    ctx.check(_lib.lqm_bdg_chemicalpotential(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(w), float(filling),
                                             float(T), float(mu_lo), float(mu_hi), ctypes.byref(out)))
    return out.value


def commutator_kspace_norm(H, rho, ks, kweights=None, multimode="cuda", ctx=None):
    """``commutator_kspace_norm(H, ρ, ks; kweights)`` (Meanfield/selfconsistent.jl:130-166):
    sqrt(sum_k w_k ||H(k) ρ(k) - ρ(k) H(k)||_F^2), w = 1/nk by default
    (``lqm_commutator_norm``)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    Rd = _as_device_hops(rho, ctx)
    ks = _ks(ks, Hd.d)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = _D()
    ctx.check(_lib.lqm_commutator_norm(ctx.handle, Hd.handle, Rd.handle, ks.shape[1], _ptr(ks), _ptr(w),
                                       ctypes.byref(out)))
    return out.value


def berry_flux(H, NX, NY, band_sets, ctx=None):
    """Summed plaquette phases of each band manifold in ``band_sets`` (lists of 0-based
    band indices) on one NX x NY state grid (``lqm_berry_flux``)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    sets = [list(map(int, s)) for s in band_sets]
    ptr = np.ascontiguousarray(np.cumsum([0] + [len(s) for s in sets]), dtype=np.int64)
    cols = np.ascontiguousarray([b for s in sets for b in s], dtype=np.int64)
    out = np.zeros(len(sets))
    ctx.check(_lib.lqm_berry_flux(ctx.handle, Hd.handle, int(NX), int(NY), len(sets), _ptr(ptr), _ptr(cols),
                                  _ptr(out)))
    return out


def berryalongpath(H, kpoints, multimode="cuda", ctx=None):
    """``berryalongpath(H, kpoints)`` (Spectrum/berry.jl:170-238): the abelian Berry
    curvature (plaquette phase) of every band at every path point, (n, N)
    (``lqm_berry_path``)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    kp = _ks(kpoints, Hd.d)
    out = np.zeros((Hd.n, kp.shape[1]), order="F")
    ctx.check(_lib.lqm_berry_path(ctx.handle, Hd.handle, kp.shape[1], _ptr(kp), _ptr(out)))
    return out


def wilson_slices(H, NX, NY=0, bands=(0,), direction=1, want_vectors=False, ctx=None):
    """The Wilson loops of WilsonSlice1D (Spectrum/berry.jl:312-367) on the statesgrid of
    ``bands`` (0-based): (en (nloops, nb), U (nloops, nb, nb) or None); direction 1 loops
    along k_y per k_x, direction 2 along k_x per k_y (``lqm_wilson``)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    NY = NX if NY < 1 else NY
    b = np.ascontiguousarray(bands, dtype=np.int64)
    nloops = (NX - 1) if direction == 1 else (NY - 1)
    en = np.zeros((nloops, len(b)))
    U = np.zeros((nloops, len(b), len(b)), dtype=np.complex128) if want_vectors else None
    Uc = np.zeros((len(b), len(b), nloops), dtype=np.complex128, order="F") if want_vectors else None
    ctx.check(_lib.lqm_wilson(ctx.handle, Hd.handle, int(NX), int(NY), len(b), _ptr(b), int(direction), _ptr(en),
                              _ptr(Uc)))
    if want_vectors:
        U = np.moveaxis(Uc, 2, 0)
    return en, U


def wilson2d(H, NX, NY=0, bands=(0,), ctx=None):
    """``Wilson2D(H, NX, NY, bandindices)`` (Spectrum/berry.jl:258-268) with 0-based bands:
    (en1, U1, en2, U2)."""
    en1, U1 = wilson_slices(H, NX, NY, bands, 1, True, ctx)
    en2, U2 = wilson_slices(H, NX, NY, bands, 2, True, ctx)
    return en1, U1, en2, U2


def wilson_wannier2d(H, NX, NY=0, bands=(0,), ctx=None):
    """``WilsonWannier2D(H, NX, NY, bandindices)`` (Spectrum/berry.jl:274-301) with 0-based
    bands: (p1, p2), the mean nested-Wilson-loop phases per band (``lqm_wilson_wannier``)."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    NY = NX if NY < 1 else NY
    b = np.ascontiguousarray(bands, dtype=np.int64)
    p1, p2 = np.zeros(len(b)), np.zeros(len(b))
    ctx.check(_lib.lqm_wilson_wannier(ctx.handle, Hd.handle, int(NX), int(NY), len(b), _ptr(b), _ptr(p1), _ptr(p2)))
    return p1, p2


def autotune_eigh(H, ks, want_rho=True, ctx=None):
    """Times every candidate block size of the one-CTA eigensolver for H's order on the
    sample k-points ``ks`` (the rho_k pass when ``want_rho``, else eigenvectors) and keeps
    the fastest on the context (``lqm_autotune_eigh``): (best_nt, best_ms, {nt: ms}).
    For an order on the blocked path the candidates are the reductions instead, 0
    (one-stage) and 1 (two-stage), kept for that order and pass kind."""
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    best, bms, nc = ctypes.c_int(), _D(), _I64()
    cnt = np.zeros(16, dtype=np.int32)
    cms = np.zeros(16)
    ctx.check(_lib.lqm_autotune_eigh(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), int(bool(want_rho)),
                                     ctypes.byref(best), ctypes.byref(bms), 16, _ptr(cnt), _ptr(cms),
                                     ctypes.byref(nc)))
    return best.value, bms.value, {int(cnt[i]): float(cms[i]) for i in range(nc.value)}


def getcherns(H, NX, NY=0, bands=None, multimode="cuda", ctx=None):
    """``getcherns(H, NX, NY, bands)`` (Spectrum/berry.jl:378-382) with 0-based band
    indices (all bands when None): the Chern number of each band, unrounded."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    NY = NX if NY < 1 else NY
    bands = list(range(Hd.n)) if bands is None else list(bands)
    return list(berry_flux(Hd, NX, NY, [[b] for b in bands], ctx=ctx))


def _berry_grid(NX, NY):
    i = np.tile(np.arange(NX), NY)
    j = np.repeat(np.arange(NY), NX)
    return np.asfortranarray(np.vstack([i / (NX - 1), j / (NY - 1)]) + 1.34e-8)


def spectralgaps(H, NX, NY=0, gaptol=1e-6, multimode="cuda", ctx=None):
    """``spectralgaps(H, NX, NY; gaptol)`` (Spectrum/berry.jl:421-442): [(n, elo, ehi)] for
    every gap wider than gaptol between the grid maximum of band n and the grid minimum of
    band n + 1 (n the number of bands below), from the device bands on the statesgrid
    k-points."""
    _check_mode(multimode)
    NY = NX if NY < 1 else NY
    E, _ = bandmatrix(H, _berry_grid(NX, NY), ctx=ctx)
    emin, emax = E.min(axis=1), E.max(axis=1)
    return [(m + 1, float(emax[m]), float(emin[m + 1])) for m in range(E.shape[0] - 1)
            if emin[m + 1] - emax[m] > gaptol]


def gapcherns(H, NX, NY=0, gaptol=1e-6, multimode="cuda", ctx=None):
    """``gapcherns(H, NX, NY; gaptol)`` (Spectrum/berry.jl:470-487): [(n, elo, ehi, chern)]
    with chern the rounded Berry flux of the lowest n bands (one state grid for all gaps)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    NY = NX if NY < 1 else NY
    gaps = spectralgaps(Hd, NX, NY, gaptol, ctx=ctx)
    if not gaps:
        return []
    flux = berry_flux(Hd, NX, NY, [list(range(m)) for m, _, _ in gaps], ctx=ctx)
    return [(m, lo, hi, int(round(f))) for (m, lo, hi), f in zip(gaps, flux)]


def fermisurfacedensity(H, energies, ks=None, broadening="auto", obs=None, num_points=15, multimode="cuda",
                        ctx=None):
    """``fermisurfacedensity(H, energies; broadening, num_points)`` (Spectrum/fermisurface.jl)
    on the device (``lqm_fermisurface``): (ks, density (nE, nk), broadening).  ``ks``
    defaults to ``regulargrid(nk=num_points^2)``; ``obs`` (n, nk) weights the bands as
    fermisurfacedensity_fromdata(bands, energies, obs) does."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    if ks is None:
        n1 = int(num_points)
        it = np.arange(n1) / n1
        ks = np.vstack([np.tile(it, n1), np.repeat(it, n1)])
    ks = _ks(ks, Hd.d)
    E = np.ascontiguousarray(np.atleast_1d(energies), dtype=np.float64)
    w = None if obs is None else np.asfortranarray(obs, dtype=np.float64)
    g = 0.0 if (broadening is None or isinstance(broadening, str)) else float(broadening)
    if not isinstance(broadening, str) and broadening is not None and not g > 0:
        raise ValueError("broadening must be positive or 'auto'")
    out = np.zeros((len(E), ks.shape[1]), order="F")
    gu = _D()
    ctx.check(_lib.lqm_fermisurface(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), len(E), _ptr(E), g, _ptr(w),
                                    _ptr(out), ctypes.byref(gu)))
    return ks, out, gu.value


def chemicalpotential(H, ks, filling, T=0.0, kweights=None, multimode="cuda", ctx=None):
    """``chemicalpotential(H, ks, filling; T)``."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    mu = _D()
    ctx.check(_lib.lqm_chemicalpotential(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(w),
                                         float(filling), float(T), ctypes.byref(mu)))
    return mu.value


def getdos(h, omegas, ks, gamma, kweights=None, multimode="cuda", ctx=None):
    """``getdos(h, ωs, ks; Γ)`` (no 1/π, divided by nk when unweighted)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(h, ctx)
    ks = _ks(ks, Hd.d)
    om = np.ascontiguousarray(omegas, dtype=np.float64)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = np.zeros(len(om))
    ctx.check(_lib.lqm_dos(ctx.handle, Hd.handle, ks.shape[1], _ptr(ks), _ptr(w), len(om), _ptr(om),
                           float(gamma), _ptr(out)))
    return out


def bands_dos_rho(rhos, H, ks, omegas, gamma, kweights=None, mu=0.0, T=0.01, multimode="cuda",
                  precision=0, ctx=None):
    """bands + DOS + ``getdensitymatrix!`` from one eigen pass (``lqm_bands_dos_rho``).
    Fills ``rhos`` in place; returns (bands (n, nk), dos (nw,), band energy)."""
    _check_mode(multimode)
    ctx = ctx or default_context()
    Hd = _as_device_hops(H, ctx)
    ks = _ks(ks, Hd.d)
    nk = ks.shape[1]
    Lkeys = list(rhos.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    om = np.ascontiguousarray(omegas, dtype=np.float64)
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    rho = np.zeros((Hd.n, Hd.n, len(Lkeys)), dtype=np.complex128, order="F")
    bands = np.zeros((Hd.n, nk), order="F")
    dos = np.zeros(len(om))
    eb = _D()
    ctx.check(_lib.lqm_bands_dos_rho(ctx.handle, Hd.handle, nk, _ptr(ks), _ptr(w), float(mu), float(T),
                                     len(Lkeys), _ptr(Lk), _ptr(rho), ctypes.byref(eb), len(om), _ptr(om),
                                     float(gamma), _ptr(dos), _ptr(bands), int(precision)))
    for i, L in enumerate(Lkeys):
        rhos[L] = np.array(rho[:, :, i])
    return bands, dos, eb.value


HFResult = namedtuple("HFResult", ["rho", "energy", "mf", "converged", "residual"])
MFInfo = namedtuple("MFInfo", ["mu", "eH", "eF", "eband", "ekin", "iterations", "eJ"], defaults=(0.0,))


class ExchangeKernel:
    """``ExchangeKernel(j, siteof, flavorof)`` (Meanfield/hartreefock.jl:24-76) with 0-based
    sites and flavors: ``j`` a site-space Hops (dict key -> ns x ns), ``siteof[I]`` and
    ``flavorof[I]`` the site and flavor of orbital I.  Validated when it is installed
    on a context."""

    def __init__(self, j, siteof, flavorof):
        self.j = {tuple(int(x) for x in L): np.asarray(M, np.complex128) for L, M in j.items()}
        self.siteof = np.ascontiguousarray(siteof, dtype=np.int64)
        self.flavorof = np.ascontiguousarray(flavorof, dtype=np.int64)
        if len(self.siteof) != len(self.flavorof):
            raise ValueError("siteof and flavorof must have equal length")

    def install(self, ctx):
        keys = list(self.j.keys())
        d = len(keys[0])
        ns = self.j[keys[0]].shape[0]
        K = np.asfortranarray(np.array(keys, dtype=np.int64).T)
        B = np.asfortranarray(np.stack([self.j[L] for L in keys], -1))
        ctx.check(_lib.lqm_ctx_set_scf_exchange(ctx.handle, ns, len(keys), d, _ptr(K), _ptr(B), len(self.siteof),
                                                _ptr(self.siteof), _ptr(self.flavorof)))


def _set_functional(ctx, hartree, fock, exchange):
    ctx.check(_lib.lqm_ctx_set_scf_terms(ctx.handle, int(bool(hartree)), int(bool(fock))))
    if exchange is None:
        ctx.check(_lib.lqm_ctx_set_scf_exchange(ctx.handle, 0, 0, 0, None, None, 0, None, None))
    else:
        exchange.install(ctx)


def hartreefock_eval(h, v, rho, hartree=True, fock=True, exchange=None, keys=None, ctx=None):
    """``hf(ρ)`` of ``HartreeFock(h, v; hartree, fock, exchange)``
    (Meanfield/hartreefock.jl:184-228,247-410) on the device (``lqm_hartreefock_eval``):
    returns (hMF dict, eH, eF, eJ); hMF on ``keys`` (default keys(h) + keys(v) + the
    exchange keys present in rho)."""
    ctx = ctx or default_context()
    _set_functional(ctx, hartree, fock, exchange)
    hd = _as_device_hops(h, ctx)
    vd = _as_device_hops(v, ctx)
    Lkeys = list(rho.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    R = np.asfortranarray(np.stack([np.asarray(rho[L], np.complex128) for L in Lkeys], -1))
    if keys is None:
        keys = list(hd.keys) if isinstance(h, DeviceHops) else [tuple(L) for L in h.keys()]
        vkeys = vd.keys if isinstance(v, DeviceHops) else [tuple(L) for L in v.keys()]
        keys += [L for L in vkeys if L not in keys]
        if exchange is not None:
            keys += [L for L in exchange.j if L in rho and L not in keys]
    keys = [tuple(L) for L in keys]
    Mk = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    out = np.zeros((hd.n, hd.n, len(keys)), dtype=np.complex128, order="F")
    en = np.zeros(3)
    ctx.check(_lib.lqm_hartreefock_eval(ctx.handle, hd.handle, vd.handle, len(Lkeys), _ptr(Lk), _ptr(R), len(keys),
                                        _ptr(Mk), _ptr(out), _ptr(en)))
    return {L: np.array(out[:, :, i]) for i, L in enumerate(keys)}, en[0], en[1], en[2]


def _hf_result(rho_out, out, mf, convergenceerror):
    """(ρ, ϵ_GS, mf, converged, residual) from lqm_scf_hf's scalars.  Not converged:
    a warning as fixedpoint! gives (Meanfield/fixedpoint.jl:189-191), and with
    ``convergenceerror`` an error (Meanfield/selfconsistent.jl:315-317)."""
    converged = bool(out[7])
    if not converged:
        warnings.warn(f"SCF stopped before reaching the tolerance; residual {out[6]} after {int(out[8])} "
                      f"iterations", stacklevel=3)
        if convergenceerror:
            raise LQMError(-5, "SCF did not converge (convergenceerror=True)")
    return HFResult(rho_out, out[0], mf, converged, out[6])


def solvehartreefock(h, v, rho_init, filling, ks, T=0.0, beta=1.0, tol=1e-7, iterations=500,
                     kweights=None, log_callback=None, multimode="cuda", ctx=None, acceleration="linear",
                     anderson_depth=5, residual_norm="density", hartree=True, fock=True, exchange=None,
                     convergenceerror=False):
    """``solvehartreefock(h, v, ρ_init, filling, ks; T, β, tol, iterations, acceleration,
    anderson_depth, residual_norm, convergenceerror)``: linear damped mixing (default) or
    Anderson acceleration; the relative density change (default) or the commutator norm
    ||[H_MF, ρ]|| as the residual.  Returns (ρ, ϵ_GS, mf, converged, residual) like the
    reference; an unconverged SCF warns, and raises with ``convergenceerror=True``."""
    _check_mode(multimode)
    acceleration = str(acceleration).lstrip(":")
    residual_norm = str(residual_norm).lstrip(":")
    if acceleration not in ("linear", "anderson"):
        raise ValueError(f"acceleration must be 'linear' or 'anderson', got {acceleration!r}")
    if residual_norm not in ("density", "commutator"):
        raise ValueError(f"residual_norm must be :density or :commutator, got {residual_norm!r}")
    ctx = ctx or default_context()
    depth = int(anderson_depth) if acceleration == "anderson" else 0
    ctx.check(_lib.lqm_ctx_set_scf_acceleration(ctx.handle, depth))
    ctx.check(_lib.lqm_ctx_set_scf_residual(ctx.handle, 1 if residual_norm == "commutator" else 0))
    _set_functional(ctx, hartree, fock, exchange)
    hd = _as_device_hops(h, ctx)
    vd = _as_device_hops(v, ctx)
    ks = _ks(ks, hd.d)
    Lkeys = list(rho_init.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    rho = np.asfortranarray(np.stack([np.asarray(rho_init[L], np.complex128) for L in Lkeys], -1))
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    out = np.zeros(9)

    def _cb(it, E, res, ekin, eband, eH, eF, mu, user):
        if log_callback is None:
            return 0
        r = log_callback(int(it), E, res, dict(ekin=ekin, eband=eband, eH=eH, eF=eF, mu=mu))
        return 1 if r is False else 0

    cb = LOG_CB(_cb)
    ctx.check(_lib.lqm_scf_hf(ctx.handle, hd.handle, vd.handle, ks.shape[1], _ptr(ks), _ptr(w),
                              float(filling), float(T), float(beta), float(tol), int(iterations),
                              len(Lkeys), _ptr(Lk), _ptr(rho), cb, None, _ptr(out)))
    rho_out = {L: np.array(rho[:, :, i]) for i, L in enumerate(Lkeys)}
    eJ = _D()
    ctx.check(_lib.lqm_ctx_scf_exchange_energy(ctx.handle, ctypes.byref(eJ)))
    mf = MFInfo(mu=out[1], eH=out[2], eF=out[3], eband=out[4], ekin=out[5], iterations=int(out[8]), eJ=eJ.value)
    return _hf_result(rho_out, out, mf, convergenceerror)


BdGMFInfo = namedtuple("BdGMFInfo", ["mu", "eH", "eF", "eP", "eband", "ekin", "iterations"])


def solvehartreefock_bdg(h, v, rho_init, filling, ks, T=0.0, beta=1.0, tol=1e-7, iterations=500,
                         log_callback=None, hartree=True, fock=True, acceleration="linear", anderson_depth=5,
                         residual_norm="density", ctx=None, convergenceerror=False):
    """``solvehartreefock(h::BdGOperator, v, ρ_init::BdGOperator, filling, ks; T, β, tol,
    iterations, convergenceerror)``: Hartree-Fock with the pairing channel (HartreeFockBDG,
    Superconductivity/hartreefock.jl:5-159) on the device (``lqm_scf_hf_bdg``).  ``h`` and
    ``v`` are the electron-sector Hops (order d), ``rho_init`` the Nambu density matrix
    (order 2d).  Returns (ρ, ϵ_GS, mf, converged, residual)."""
    ctx = ctx or default_context()
    acceleration = str(acceleration).lstrip(":")
    residual_norm = str(residual_norm).lstrip(":")
    if acceleration not in ("linear", "anderson"):
        raise ValueError(f"acceleration must be 'linear' or 'anderson', got {acceleration!r}")
    if residual_norm not in ("density", "commutator"):
        raise ValueError(f"residual_norm must be :density or :commutator, got {residual_norm!r}")
    ctx.check(_lib.lqm_ctx_set_scf_acceleration(ctx.handle, int(anderson_depth) if acceleration == "anderson" else 0))
    ctx.check(_lib.lqm_ctx_set_scf_residual(ctx.handle, 1 if residual_norm == "commutator" else 0))
    _set_functional(ctx, hartree, fock, None)
    hd = _as_device_hops(h, ctx)
    vd = _as_device_hops(v, ctx)
    ks = _ks(ks, hd.d)
    Lkeys = list(rho_init.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    rho = np.asfortranarray(np.stack([np.asarray(rho_init[L], np.complex128) for L in Lkeys], -1))
    out = np.zeros(10)

    def _cb(it, E, res, ekin, eband, eH, eF, mu, user):
        if log_callback is None:
            return 0
        r = log_callback(int(it), E, res, dict(ekin=ekin, eband=eband, eH=eH, eF=eF, mu=mu))
        return 1 if r is False else 0

    cb = LOG_CB(_cb)
    ctx.check(_lib.lqm_scf_hf_bdg(ctx.handle, hd.handle, vd.handle, ks.shape[1], _ptr(ks), float(filling), float(T),
                                  float(beta), float(tol), int(iterations), len(Lkeys), _ptr(Lk), _ptr(rho), cb, None,
                                  _ptr(out)))
    rho_out = {L: np.array(rho[:, :, i]) for i, L in enumerate(Lkeys)}
    mf = BdGMFInfo(mu=out[1], eH=out[2], eF=out[3], eP=out[9], eband=out[4], ekin=out[5], iterations=int(out[8]))
    return _hf_result(rho_out, out, mf, convergenceerror)


SCFGradient = namedtuple("SCFGradient", ["F", "omega", "N", "dF_dh", "dL_dh", "residual", "iterations"])


def scf_hf_gradient(h, v, rho, mu, ks, T=0.0, kweights=None, eps_bar=None, beta=0.3, tol=1e-12, iterations=2000,
                    hartree=True, fock=True, ctx=None):
    """Derivatives of a converged Hartree-Fock SCF (``lqm_scf_hf_gradient``): the free
    energy F of hMF = hf(rho) at mu, dF/dh_R (the density matrix of hMF at the keys of h),
    and, with ``eps_bar`` (n, nk) the cotangent of the mean-field bands, the total
    dL/dh_R through the fixed point.  ``rho`` and ``mu`` are the converged density
    matrix and chemical potential (``solvehartreefock`` with the same ks, T, weights).
    Gradients are dicts keyed like h, paired as dL = Re sum_R <G_R, dh_R>."""
    ctx = ctx or default_context()
    _set_functional(ctx, hartree, fock, None)
    hd = _as_device_hops(h, ctx)
    vd = _as_device_hops(v, ctx)
    ks = _ks(ks, hd.d)
    nk = ks.shape[1]
    Lkeys = list(rho.keys())
    Lk = np.asfortranarray(np.array(Lkeys, dtype=np.int64).T)
    R = np.asfortranarray(np.stack([np.asarray(rho[L], np.complex128) for L in Lkeys], -1))
    w = None if kweights is None else np.ascontiguousarray(kweights, dtype=np.float64)
    hkeys = list(hd.keys) if isinstance(h, DeviceHops) else [tuple(k) for k in h.keys()]
    dF = np.zeros((hd.n, hd.n, len(hkeys)), dtype=np.complex128, order="F")
    eb = None if eps_bar is None else np.asfortranarray(np.asarray(eps_bar, dtype=np.float64))
    dL = np.zeros_like(dF) if eb is not None else None
    out = np.zeros(5)
    ctx.check(_lib.lqm_scf_hf_gradient(ctx.handle, hd.handle, vd.handle, nk, _ptr(ks), _ptr(w), float(T), float(mu),
                                       len(Lkeys), _ptr(Lk), _ptr(R), _ptr(eb), float(beta), float(tol),
                                       int(iterations), _ptr(dF), _ptr(dL), _ptr(out)))
    dFd = {Rk: np.array(dF[:, :, i]) for i, Rk in enumerate(hkeys)}
    dLd = None if dL is None else {Rk: np.array(dL[:, :, i]) for i, Rk in enumerate(hkeys)}
    return SCFGradient(out[0], out[1], out[2], dFd, dLd, out[3], int(out[4]))


def bands_dos_rho_multi_dev(models, d_ks, nk, mu=0.0, T=0.01, gamma=0.05, d_w=None, ctx=None):
    """``lqm_bands_dos_rho_multi_dev``: bands, DOS and rho_L of several models on one k list
    (device arrays) with ONE eigensolver launch.  ``models``: list of dicts with
    ``H`` (DeviceHops), ``Lk`` (keys d x nL int64, F order), ``rho`` (device nL x n x n
    complex), ``om`` (device omegas), ``dos`` (device nw), ``bands`` (device nk x n).
    Returns the band energies."""
    ctx = ctx or default_context()
    nm = len(models)
    arr = ctypes.c_void_p * nm
    Hs = arr(*[m["H"].handle.value if isinstance(m["H"].handle, ctypes.c_void_p) else m["H"].handle for m in models])
    nL = np.array([m["Lk"].shape[1] for m in models], dtype=np.int64)
    Lk = arr(*[m["Lk"].ctypes.data for m in models])
    rho = arr(*[m["rho"].data_ptr() for m in models])
    om = arr(*[m["om"].data_ptr() for m in models])
    dos = arr(*[m["dos"].data_ptr() for m in models])
    bands = arr(*[m["bands"].data_ptr() for m in models])
    eb = np.zeros(nm)
    nw = int(models[0]["om"].numel())
    ctx.check(_lib.lqm_bands_dos_rho_multi_dev(ctx.handle, nm, ctypes.cast(Hs, _P), int(nk), _ptr(d_ks), _ptr(d_w),
                                               float(mu), float(T), _ptr(nL), ctypes.cast(Lk, _P),
                                               ctypes.cast(rho, _P), _ptr(eb), nw, ctypes.cast(om, _P), float(gamma),
                                               ctypes.cast(dos, _P), ctypes.cast(bands, _P)))
    return eb
