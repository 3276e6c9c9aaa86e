"""The allocation-free eigen pass agrees with the regular entry point.

``lqm_bandmatrix_noalloc`` serves callers that cannot allocate device memory
(a host whose device memory belongs to another allocator, such as a Julia
CUDA.jl pool or a framework's caching allocator, or a latency-sensitive loop
that cannot afford cudaMalloc's device-wide synchronisation).  It takes only
caller-owned device buffers and uses a fixed device array inside the library
for scratch.  This test owns the buffers (torch allocations on the test side),
calls the entry point twice in a row through the C-ABI, checks that the second
call leaves the device's free memory unchanged, and compares both
results with ``lqm_bandmatrix_dev`` at the band tolerance used elsewhere
(1e-10 of the spectral width) and the eigenvectors to 1e-12.  The regular
call runs on a context held to the same one-CTA-per-k eigensolver, so the two
produce the same eigenvector phases.
"""
import ctypes

import numpy as np
import pytest

from lqm_workloads import lattice as L
from lqm_workloads import models as M

pytestmark = pytest.mark.gpu
BAND_TOL = 1e-10


def _cases():
    return [("triangular4x4_soc n=96 (shared-memory path)", M.batch_models()[2][1]),
            ("honeycomb 6x6 n=144 (global-scratch path)", M.honeycomb_disorder()[1])]


@pytest.fixture(scope="module")
def ctx1(lqm):
    """A context held to the one-CTA-per-k eigensolver (the path the allocation-free
    entry point uses) at every order that fits it."""
    c = lqm.Context(0, timeout=600)
    c.set_blocked_min_n(10 ** 9)
    yield c
    c.close()


@pytest.mark.parametrize("name,h", _cases(), ids=["n96", "n144"])
def test_noalloc_matches_regular_entry_point(lqm, ctx1, name, h):
    import torch
    ctx = ctx1
    dev = torch.device("cuda", 0)
    n, nR, d, K, B = lqm.pack_hops(h)
    ks = np.hstack([L.regulargrid(12 * 12), np.random.default_rng(1).random((2, 56))])
    nk = ks.shape[1]
    d_keys = torch.from_numpy(np.ascontiguousarray(K.T)).to(dev)             # d x nR column-major
    d_blocks = torch.from_numpy(np.ascontiguousarray(B.transpose(2, 1, 0))).to(dev)  # n x n x nR column-major
    d_ks = torch.from_numpy(np.ascontiguousarray(ks.T)).to(dev)
    ref_b = torch.zeros(nk, n, dtype=torch.float64, device=dev)
    ref_U = torch.zeros(nk, n, n, dtype=torch.complex128, device=dev)
    Hd = lqm.DeviceHops(h, ctx)
    ctx.check(lqm.lib().lqm_bandmatrix_dev(ctx.handle, Hd.handle, nk, lqm._ptr(d_ks), 1, 0, lqm._ptr(ref_b),
                                           lqm._ptr(ref_U)))
    ref_b, ref_U = ref_b.cpu().numpy(), ref_U.cpu().numpy()
    scale = ref_b.max() - ref_b.min()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        b = torch.full((nk, n), float("nan"), dtype=torch.float64, device=dev)
        U = torch.full((nk, n, n), float("nan"), dtype=torch.complex128, device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        st = lqm.lib().lqm_bandmatrix_noalloc(stream, n, nR, d, lqm._ptr(d_keys), lqm._ptr(d_blocks), nk,
                                              lqm._ptr(d_ks), lqm._ptr(b), lqm._ptr(U))
        assert st == 0, (name, call, st)
        torch.cuda.synchronize()
        if call == 1:  # after the first call's one-time set-up, a call takes no device memory at all
            assert torch.cuda.mem_get_info(dev)[0] == free_before, (name, call)
        b, U = b.cpu().numpy(), U.cpu().numpy()
        assert np.max(np.abs(b - ref_b)) <= BAND_TOL * scale, (name, call)
        assert np.max(np.abs(U - ref_U)) <= 1e-12, (name, call)


def test_noalloc_rejects_sizes_beyond_its_limit(lqm):
    # n above the 1024 limit is refused before any device work
    st = lqm.lib().lqm_bandmatrix_noalloc(None, 1025, 1, 2, ctypes.c_void_p(8), ctypes.c_void_p(8), 1,
                                          ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert st == -1
