"""World-size-2 CPU (gloo) check of the multi-GPU decomposition used by bench.py.

Each rank takes its slice of the k grid (bench.kgrid), computes rho_L and the DOS
of its slice with uniform weights 1/nk_local, and the ranks combine them with
bench.reduce_shards (all-reduce sum / world).  The result must equal the
single-process result on the union grid.  The oracle stands in for the per-rank
device computation; the sharding and the collective are what is tested.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "latticeqm.jl_b200", "python")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from lqm_workloads import models as M
    from oracle import kspace as K
    h = M.batch_models()[0][1]
    ks = bench.kgrid(rank, world, nk_lin=4)
    nk = ks.shape[1]
    w = np.full(nk, 1.0 / nk)
    rho, _ = K.densitymatrix(h, ks, w, 0.0, 0.01, list(h.keys()))
    b, _ = K.bandmatrix(h, ks)
    om = np.linspace(-4, 4, 50)
    dos = K.dos_from_bands(b, om, 0.05)
    t_rho = torch.from_numpy(np.stack([rho[R] for R in h]))
    t_dos = torch.from_numpy(dos)
    bench.reduce_shards(dist, (t_rho, t_dos), world)
    if rank == 0:
        np.save(os.path.join(out_dir, "rho.npy"), t_rho.numpy())
        np.save(os.path.join(out_dir, "dos.npy"), t_dos.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_reproduce_the_full_grid(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "latticeqm.jl_b200", "python")]
    import bench
    from lqm_workloads import models as M
    from oracle import kspace as K
    h = M.batch_models()[0][1]
    full = np.hstack([bench.kgrid(r, world, nk_lin=4) for r in range(world)])
    # the union of the slices is the (4*world) x 4 grid, each k once
    assert len({tuple(np.round(k, 12)) for k in full.T}) == full.shape[1] == 4 * world * 4
    w = np.full(full.shape[1], 1.0 / full.shape[1])
    rho, _ = K.densitymatrix(h, full, w, 0.0, 0.01, list(h.keys()))
    b, _ = K.bandmatrix(h, full)
    dos = K.dos_from_bands(b, np.linspace(-4, 4, 50), 0.05)
    got_rho = np.load(tmp_path / "rho.npy")
    got_dos = np.load(tmp_path / "dos.npy")
    assert np.max(np.abs(got_rho - np.stack([rho[R] for R in h]))) < 1e-13
    assert np.max(np.abs(got_dos - dos)) < 1e-12
