"""Several models of uneven order in one eigensolver launch (lqm_bands_dos_rho_multi_dev).

The batched workload's three models (square 2x2 n = 8, kagome 2x2 n = 24, triangular
4x4 with spin-orbit phases n = 96) on one k list: each model's k-points run on CTA
sub-teams of that model's one-CTA block size (12 teams of 32 threads, 6 of 64, or
the whole 384-thread CTA) within ONE kernel launch.  The per-k code and team sizes
are those of the per-model launches, so the bands must be bit-identical to
lqm_bands_dos_rho_dev model by model; rho_L, the DOS and the band energy (whose
k-sums are chunked differently) agree to 1e-12, and everything agrees with the
oracle at the tolerances of the other parity tests."""
import ctypes

import numpy as np
import pytest

from oracle import kspace as K
from lqm_workloads import lattice as L
from lqm_workloads import models as M

pytestmark = pytest.mark.gpu
NW, GAMMA, MU, TEMP = 64, 0.05, 0.0, 0.01


def _state(lqm, ctx, torch, dev, h, nk):
    Hd = lqm.DeviceHops(h, ctx)
    n = Hd.n
    return dict(H=Hd, h=h, n=n, Lk=np.asfortranarray(np.array(list(h.keys()), dtype=np.int64).T),
                rho=torch.zeros(len(h), n, n, dtype=torch.complex128, device=dev),
                dos=torch.zeros(NW, dtype=torch.float64, device=dev),
                om=torch.linspace(-5.0, 5.0, NW, dtype=torch.float64, device=dev),
                bands=torch.zeros(nk, n, dtype=torch.float64, device=dev))


def test_one_launch_matches_per_model_launches_and_oracle(lqm, ctx):
    import torch
    dev = torch.device("cuda", 0)
    ks = np.hstack([L.regulargrid(48 * 48), np.random.default_rng(4).random((2, 37))])
    nk = ks.shape[1]
    d_ks = torch.from_numpy(np.ascontiguousarray(ks.T)).to(dev)
    models = [h for _, h in M.batch_models()]
    one = [_state(lqm, ctx, torch, dev, h, nk) for h in models]
    ctx.reset_stats(timing=True)
    eb1 = lqm.bands_dos_rho_multi_dev(one, d_ks, nk, mu=MU, T=TEMP, gamma=GAMMA, ctx=ctx)
    _, eigh_launches, _ = ctx.stats()
    assert eigh_launches == 1  # every model's k-points in one eigensolver launch
    eb = ctypes.c_double()
    for s, e1 in zip(one, eb1):
        ref = _state(lqm, ctx, torch, dev, s["h"], nk)
        ctx.check(lqm.lib().lqm_bands_dos_rho_dev(
            ctx.handle, ref["H"].handle, nk, lqm._ptr(d_ks), None, MU, TEMP, ref["Lk"].shape[1], lqm._ptr(ref["Lk"]),
            lqm._ptr(ref["rho"]), ctypes.byref(eb), NW, lqm._ptr(ref["om"]), GAMMA, lqm._ptr(ref["dos"]),
            lqm._ptr(ref["bands"]), 0))
        assert torch.equal(s["bands"], ref["bands"]), s["n"]
        assert float((s["rho"] - ref["rho"]).abs().max()) <= 1e-12, s["n"]
        assert float((s["dos"] - ref["dos"]).abs().max()) <= 1e-12 * float(ref["dos"].abs().max()), s["n"]
        assert abs(e1 - eb.value) <= 1e-12 * max(1.0, abs(eb.value)), s["n"]
    # the oracle on a subset of the k-points of the smallest grid
    sub = np.arange(0, nk, 97)
    for s in one:
        b_ref, _ = K.bandmatrix(s["h"], ks[:, sub])
        b = s["bands"].cpu().numpy().T[:, sub]
        assert np.max(np.abs(b - b_ref)) / max(b_ref.max() - b_ref.min(), 1.0) <= 1e-10, s["n"]
    small = [_state(lqm, ctx, torch, dev, h, 36) for h in models]
    ks2 = L.regulargrid(6 * 6)
    d_ks2 = torch.from_numpy(np.ascontiguousarray(ks2.T)).to(dev)
    eb2 = lqm.bands_dos_rho_multi_dev(small, d_ks2, 36, mu=MU, T=TEMP, gamma=GAMMA, ctx=ctx)
    w = np.full(36, 1.0 / 36)
    for s, e2 in zip(small, eb2):
        keys = list(s["h"].keys())
        rref, ebref = K.densitymatrix(s["h"], ks2, w, MU, TEMP, keys)
        got = s["rho"].cpu().numpy()  # block i holds rho_L column-major, i.e. its transpose row-major
        assert max(np.max(np.abs(got[i].T - rref[R])) for i, R in enumerate(keys)) <= 1e-9, s["n"]
        assert abs(e2 - ebref) <= 1e-9 * max(1.0, abs(ebref)), s["n"]
