"""The C-ABI library builds, loads and exports every entry point include/kspace.h declares.

No compute call is made here: this file runs without a GPU.
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "kspace.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lqm_\w+)\s*\(", text)) - {"lqm_scf_log_cb"})


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["lqm_ctx_create", "lqm_bandmatrix", "lqm_densitymatrix", "lqm_chemicalpotential", "lqm_dos",
              "lqm_scf_hf", "lqm_hops_upload_dense", "lqm_hops_upload_csc", "lqm_bloch"]:
        assert s in syms


def test_library_exports_every_declared_symbol(lqm):
    lib = lqm.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(lqm.EXPORTS) == set(declared_symbols())


def test_null_arguments_are_rejected_without_a_device(lqm):
    lib = lqm.lib()
    assert lib.lqm_ctx_create(0, None) == -1          # LQM_EINVAL
    assert lib.lqm_ctx_destroy(None) == -1
    assert lib.lqm_hops_free(None, None) == -1
    assert lib.lqm_last_error(None) == b"null context"


def test_context_creation_reports_missing_device(lqm):
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    st = lqm.lib().lqm_ctx_create(0, ctypes.byref(h))
    assert st == -2 and not h.value                   # LQM_ECUDA, no CPU fallback


def test_pack_hops_layout(lqm):
    """pack_hops hands the C-ABI the layout lqm_hops_upload_dense reads: keys d x nR
    and blocks n x n x nR, both column-major (Julia's), block r = h[key r]."""
    import numpy as np
    rng = np.random.default_rng(4)
    h = {(i, j): rng.normal(size=(5, 5)) + 1j * rng.normal(size=(5, 5)) for i in (-1, 0, 1) for j in (0, 2)}
    n, nR, d, K, B = lqm.pack_hops(h)
    assert (n, nR, d) == (5, 6, 2)
    assert K.dtype == np.int64 and K.flags.f_contiguous and K.shape == (2, 6)
    assert B.dtype == np.complex128 and B.flags.f_contiguous and B.shape == (5, 5, 6)
    flat = np.frombuffer(B.tobytes(order="A"), dtype=np.complex128)
    for r, R in enumerate(h):
        assert tuple(K[:, r]) == R
        # column-major block r starts at r * n * n; element (i, j) at i + j * n
        blk = flat[r * 25:(r + 1) * 25].reshape(5, 5, order="F")
        assert np.array_equal(blk, h[R])


def test_empty_kset_matches_oracle_without_a_device(lqm):
    """An empty k-set gives what the reference's loops give when they run zero times
    (bands.jl:164-204, densitymatrix.jl:17-49): n x 0 bands, zeroed rho blocks and a
    band energy of 0.  The mirror answers before any device work, so this holds on a
    machine without a GPU as well."""
    import numpy as np
    from oracle import kspace as K
    t = np.array([[0.1, 0.2], [0.0, 0.1]], complex)
    h = {(0, 0): np.diag([0.3, -0.2]).astype(complex), (1, 0): t, (-1, 0): t.conj().T}
    ks = np.zeros((2, 0))
    b, U = lqm.bandmatrix(h, ks)
    assert b.shape == K.bandmatrix(h, ks)[0].shape == (2, 0) and U is None
    b, U = lqm.bandmatrix(h, ks, want_vectors=True)
    assert b.shape == (2, 0) and U.shape == (2, 2, 0)
    bp, _ = lqm.bandmatrix(h, ks, format="sparse", num_bands=1)
    assert bp.shape == (1, 0)
    rho = {(0, 0): np.ones((2, 2), complex), (1, 0): None}
    eb = lqm.getdensitymatrix(rho, h, ks, mu=0.0, T=0.01)
    ref, eb_ref = K.densitymatrix(h, ks, np.zeros(0), 0.0, 0.01, list(rho.keys()))
    assert eb == eb_ref == 0.0
    for R in rho:
        assert np.array_equal(rho[R], ref[R]) and not rho[R].any()


def test_scf_nonconvergence_warns_and_raises(lqm):
    """An unconverged SCF warns (fixedpoint.jl:189-191) and, with convergenceerror,
    raises LQM_ENOCONV (selfconsistent.jl:315-317); a converged one does neither.
    out = lqm_scf_hf's scalars {E_GS, mu, eH, eF, eband, ekin, residual, converged, iterations}."""
    import warnings
    import pytest
    out = [-1.5, 0.1, 0.2, -0.3, -1.0, -0.8, 0.25, 0.0, 3.0]
    with pytest.warns(UserWarning, match="residual 0.25 after 3"):
        r = lqm._hf_result({}, out, None, False)
    assert r.converged is False and r.residual == 0.25 and r[1] == -1.5
    with pytest.warns(UserWarning), pytest.raises(lqm.LQMError) as err:
        lqm._hf_result({}, out, None, True)
    assert err.value.status == -5
    out[7] = 1.0
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        assert lqm._hf_result({}, out, None, True).converged is True


def test_shard_ranges_tile_the_k_list_without_a_device(lqm):
    """lqm_shard_range (host code of the multi-GPU sharding): contiguous shares that
    tile [0, nk) in rank order, sizes differing by at most one; empty shares when
    nk < nranks; invalid arguments rejected."""
    for nk in (0, 1, 3, 7, 576, 1000003):
        for nr in (1, 2, 3, 8):
            spans = [lqm.shard_range(nk, nr, r) for r in range(nr)]
            assert spans[0][0] == 0 and spans[-1][1] == nk
            assert all(spans[i][1] == spans[i + 1][0] for i in range(nr - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 0
    with pytest.raises(lqm.LQMError):
        lqm.shard_range(10, 2, 2)
    with pytest.raises(lqm.LQMError):
        lqm.shard_range(-1, 2, 0)


def test_comm_unique_id_without_a_device(lqm):
    """NCCL loads at run time and makes a communicator id (no device needed)."""
    uid = lqm.comm_unique_id()
    assert isinstance(uid, bytes) and len(uid) == lqm.COMM_ID_BYTES == 128
    assert lqm.comm_unique_id() != uid
