"""World-size-2 CPU (gloo) checks of the library's k-point sharding.

With a communicator on its context, the library splits the k list a caller passes
into contiguous shares (``lqm_shard_range``, exported host code, called here through
the C-ABI without a device), sums rho_L and the band energy over the ranks and gathers
the bands (so every rank computes the same mu), and runs the Hartree-Fock SCF with
those two exchanges per iteration and the mixing replicated.  These tests run that
decomposition on two gloo ranks, with the oracle standing in for each rank's device
pass, and compare it with the serial oracle:

* rho_L, the band energy and mu of a sharded pass equal the single-process values
  (src/modules/Parallel/Parallel.jl:275-287,415-467 is the reference's distributed
  k-loop this replaces);
* the sharded SCF (the structure of lqm_scf_hf with a communicator) follows the serial
  oracle SCF (src/modules/Meanfield/selfconsistent.jl:256-336) iteration by iteration.
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _paths():
    import sys
    for p in (ROOT, os.path.join(ROOT, "latticeqm.jl_b200", "python")):
        if p not in sys.path:
            sys.path.insert(0, p)


def _init(rank, world, port):
    _paths()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OPENBLAS_NUM_THREADS="1")
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _gather_k(arr_local, k0, k1, nk, world):
    """Every rank's block of a per-k array (k-points along the last axis) on every rank,
    as the library's grouped broadcasts leave it."""
    import lqm_cuda as Q
    shape = arr_local.shape[:-1]
    full = torch.zeros(*shape, nk, dtype=torch.float64)
    full[..., k0:k1] = torch.from_numpy(arr_local)
    for r in range(world):
        a, b = Q.shard_range(nk, world, r)
        blk = full[..., a:b].contiguous()
        dist.broadcast(blk, src=r)
        full[..., a:b] = blk
    return full.numpy()


def _allreduce(x):
    t = torch.from_numpy(np.ascontiguousarray(x))
    dist.all_reduce(t)
    return t.numpy()


def _pass_main(rank, world, port, out_dir):
    _init(rank, world, port)
    import lqm_cuda as Q
    from lqm_workloads import lattice as L
    from lqm_workloads import models as M
    from oracle import kspace as K
    h = M.batch_models()[1][1]  # kagome 2x2 spinful, n = 24
    ks = L.regulargrid(5 * 5)   # 25 k-points: uneven shares
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk)   # the full list's weights on every rank
    k0, k1 = Q.shard_range(nk, world, rank)
    keys = list(h.keys())
    rho, eb = K.densitymatrix(h, ks[:, k0:k1], w[k0:k1], 0.0, 0.01, keys)
    rho_all = _allreduce(np.stack([rho[R] for R in keys]))
    eb_all = float(_allreduce(np.array([eb]))[0])
    bands = _gather_k(K.bandmatrix(h, ks[:, k0:k1])[0], k0, k1, nk, world)
    mu = K.chemicalpotential(bands, 0.5, 0.01)
    np.savez(os.path.join(out_dir, f"pass{rank}.npz"), rho=rho_all, eb=eb_all, mu=mu, k0=k0, k1=k1)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_reproduce_the_serial_pass(tmp_path):
    world = 2
    mp.start_processes(_pass_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    _paths()
    import lqm_cuda as Q
    from lqm_workloads import lattice as L
    from lqm_workloads import models as M
    from oracle import kspace as K
    h = M.batch_models()[1][1]
    ks = L.regulargrid(25)
    nk = ks.shape[1]
    keys = list(h.keys())
    rho, eb = K.densitymatrix(h, ks, np.full(nk, 1.0 / nk), 0.0, 0.01, keys)
    mu = K.chemicalpotential(K.bandmatrix(h, ks)[0], 0.5, 0.01)
    got = [np.load(tmp_path / f"pass{r}.npz") for r in range(world)]
    # the shares tile the list: [0, 12) and [12, 25)
    assert [(int(g["k0"]), int(g["k1"])) for g in got] == [Q.shard_range(nk, world, r) for r in range(world)]
    assert int(got[0]["k0"]) == 0 and int(got[-1]["k1"]) == nk and int(got[0]["k1"]) == int(got[1]["k0"])
    for g in got:
        assert np.max(np.abs(g["rho"] - np.stack([rho[R] for R in keys]))) < 1e-13
        assert abs(float(g["eb"]) - eb) < 1e-13
        assert float(g["mu"]) == mu  # the same gathered bands give the same bisection


def _scf_main(rank, world, port, out_dir, iters):
    _init(rank, world, port)
    import lqm_cuda as Q
    from lqm_workloads import lattice as L
    from lqm_workloads import models as M
    from oracle import kspace as K
    from oracle import meanfield as MF
    lat, h, v = M.triangular_hubbard(L_super=2)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=5)}
    ks = L.regulargrid(7 * 7)
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk)
    k0, k1 = Q.shard_range(nk, world, rank)
    T, beta, filling = 0.02, 0.3, 0.5
    hf = MF.HartreeFock(h, v)
    keys = list(rho0.keys())
    residuals = []
    for _ in range(iters):  # lqm_scf_hf's iteration with a communicator
        hf(rho0)
        bands = _gather_k(K.bandmatrix(hf.hMF, ks[:, k0:k1])[0], k0, k1, nk, world)
        mu = K.chemicalpotential(bands, filling, T)
        part, eb = K.densitymatrix(hf.hMF, ks[:, k0:k1], w[k0:k1], mu, T, keys)
        rho1 = dict(zip(keys, _allreduce(np.stack([part[L_] for L_ in keys]))))
        eb = float(_allreduce(np.array([eb]))[0])
        for L_ in keys:  # linear mixing, replicated
            rho1[L_] = beta * rho1[L_] + (1 - beta) * rho0[L_]
        diff = np.linalg.norm([np.linalg.norm(rho1[L_] - rho0[L_]) for L_ in keys])
        nrm = np.linalg.norm([np.linalg.norm(rho1[L_]) for L_ in keys])
        residuals.append(diff / nrm)
        rho0 = {L_: rho1[L_].copy() for L_ in keys}
    hf(rho0)
    E = eb - hf.doublecounting()
    np.savez(os.path.join(out_dir, f"scf{rank}.npz"), rho=rho0[(0, 0)], mu=mu, E=E, res=np.array(residuals))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_scf_matches_serial_oracle(tmp_path):
    world, iters = 2, 6
    mp.start_processes(_scf_main, args=(world, _free_port(), str(tmp_path), iters), nprocs=world,
                       start_method="spawn")
    _paths()
    from lqm_workloads import lattice as L
    from lqm_workloads import models as M
    from oracle import meanfield as MF
    lat, h, v = M.triangular_hubbard(L_super=2)
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=5)}
    ks = L.regulargrid(49)
    log = []
    rho, E, hf, conv, resid, it = MF.solvehartreefock(h, v, rho0, 0.5, ks, T=0.02, beta=0.3, tol=0.0,
                                                      iterations=iters, log=lambda *a: log.append(a))
    assert it == iters
    for r in range(world):
        g = np.load(tmp_path / f"scf{r}.npz")
        assert np.max(np.abs(g["rho"] - rho[(0, 0)])) < 1e-12
        assert abs(float(g["mu"]) - hf.mu) < 1e-12
        assert abs(float(g["E"]) - E) < 1e-11
        assert np.max(np.abs(g["res"] - np.array([a[2] for a in log]))) < 1e-11
