"""Throughput of the LatticeQM k-space hot path, H(k) + eigh + rho_R, on B200.

One step = one density-matrix pass of the twisted-bilayer workload: the
commensurate twisted bilayer honeycomb (m = 10, r = 1; n = 1324 pz orbitals,
spinless) with Slater-Koster hopping (Vpp_pi = -2.7, Vpp_sigma = 0.48, decay
0.184 a, cutoff 3 a), its 24 x 24 k-grid per GPU through
``lqm_densitymatrix_dev``: Bloch sum, FP64 Hermitian eigendecomposition with
vectors (batched blocked reduction + divide and conquer + back-transformation),
rho_k = U f U^H and the Fourier fold into rho_L for the 7 keys of H (mu = 0,
T = 0.01), and the band energy.  Seeded synthetic model (no dataset exists for
this path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

Prints one JSON line on rank 0.  ``value`` is the device-resident throughput
(inputs on the device before the timed region); ``e2e`` is the same step
through the host-pointer C-ABI from pinned host memory (H uploaded, rho_L copied
back, every step).  ``--impl reference`` times the reference's :multithreaded
k-loop restated in C++/OpenMP (oracle/cpu_kspace.cpp: zheevr + zgemm + fold per
k-point, one BLAS thread per host thread) on a bounded sample of the same grid.
"""
import argparse
import ctypes
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
import warnings

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_PY = os.path.join(ROOT, "latticeqm.jl_b200", "python")
for _p in (ROOT, PKG_PY):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "k-pts/s H(k)+eigh+rho_R (FP64 plain), twisted bilayer m=10 (n=1324)"
NK_SIDE = 24
MU, TEMP = 0.0, 0.01
WORKLOAD = ("tbg_m10_n1324: twisted bilayer honeycomb (m=10, r=1; n=1324 pz orbitals, spinless), Slater-Koster "
            "Vpp_pi=-2.7, Vpp_sigma=0.48, decay 0.184a, cutoff 3a; 24x24 k-grid per GPU; rho_R for the 7 keys "
            "of H (mu=0, T=0.01) + band energy")
# the batched three-model workload, reported among the other configurations
NK_LIN = 256
NW = 500
GAMMA = 0.05
BATCH_WORKLOAD = ("batch3: square2x2 (n=8) + kagome2x2 (n=24) + triangular4x4 3-site SOC (n=96), "
                  "256x256 k-grid each; bands + DOS(500, Gamma=0.05) + rho_R (9 keys, mu=0, T=0.01)")
FALLBACK_HBM_GBS = 6650.0


def flops_per_k(n, nR, nL):
    """Algorithmic real flops per k: H(k) build, eigh with vectors, rho_k, Fourier fold."""
    return 8.0 * nR * n * n + (16.0 / 3.0 + 8.0) * n ** 3 + 4.0 * n ** 3 + 8.0 * nL * n * n


def eigh_flops_per_k(n, nR):
    return 8.0 * nR * n * n + (16.0 / 3.0 + 8.0) * n ** 3


def kgrid(rank, world, nk_lin=NK_LIN):
    """Rank r's nk_lin x nk_lin slice of a (nk_lin*world) x nk_lin grid (first index
    fastest): rank r takes the k1 values (i*world + r)/(nk_lin*world)."""
    import numpy as np
    n1 = nk_lin * world
    i = np.arange(nk_lin) * world + rank
    kx = np.tile(i / n1, nk_lin)
    ky = np.repeat(np.arange(nk_lin) / nk_lin, nk_lin)
    return np.asfortranarray(np.vstack([kx, ky]))


def full_grid(world, side=NK_SIDE):
    """The (side*world) x side grid whose k-points all ranks pass to the library; with a
    communicator set the library processes rank r's contiguous share (side x side
    points) and sums rho_L over the ranks."""
    import numpy as np
    n1 = side * world
    kx = np.tile(np.arange(n1) / n1, side)
    ky = np.repeat(np.arange(side) / side, n1)
    return np.asfortranarray(np.vstack([kx, ky]))


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json, else the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        for key in ("hbm_gbs", "hbm_GBs", "hbm"):
            if key in d:
                v = d[key]
                v = v.get("burst", v.get("value")) if isinstance(v, dict) else v
                return float(v), "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)"
    except Exception:
        pass
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU legs
def cpu_threads():
    return os.cpu_count() or 1


def cpu_density_sample(h, ks_all, start, count, threads, packed=None):
    """The oracle's C++/OpenMP density-matrix k-loop (oracle/cpu_kspace.cpp) on `count`
    consecutive points of the grid from `start` (cyclic): (k-points, seconds)."""
    import numpy as np
    from oracle import cpu as C
    nk = ks_all.shape[1]
    idx = (start + np.arange(count)) % nk
    ks = np.ascontiguousarray(ks_all[:, idx])
    t0 = time.perf_counter()
    C.densitymatrix(h, ks, None, MU, TEMP, list(h.keys()), nthreads=threads, packed=packed)
    return count, time.perf_counter() - t0


def cpu_baseline_tbg(h, ks_all, threads):
    """cpu_baseline of the headline: 2 k-points per host thread of the 24 x 24 grid."""
    from oracle import cpu as C
    pk = C._pack(h)
    cpu_density_sample(h, ks_all, 0, threads, threads, pk)  # warm (allocation, thread pool)
    done, sec = cpu_density_sample(h, ks_all, threads, 2 * threads, threads, pk)
    return {"value": done / sec, "unit": "k-pts/s", "cores": threads, "kind": "port",
            "sample": f"{done} consecutive k-points of the 24x24 grid, C++/OpenMP restatement of the "
                      f":multithreaded k-loop (per k: H(k), LAPACK zheevr, zgemm rho_k, fold into 7 keys) on "
                      f"{threads} threads, one BLAS thread each; {sec:.1f} s"}


def cpu_rate(h, ks_all, threads, per_thread=1, bands_only=False):
    """Host k-points per second of the C++ restatement on a bounded sample."""
    import numpy as np
    from oracle import cpu as C
    pk = C._pack(h)
    count = max(1, per_thread * threads)
    ks = np.ascontiguousarray(ks_all[:, np.arange(count) % ks_all.shape[1]])
    t0 = time.perf_counter()
    if bands_only:
        C.bandmatrix(h, ks, nthreads=threads, packed=pk)
    else:
        C.densitymatrix(h, ks, None, MU, TEMP, list(h.keys()), nthreads=threads, packed=pk)
    return count / (time.perf_counter() - t0)


def run_reference(args, rank, world):
    """--impl reference: LatticeQM's :multithreaded density-matrix k-loop restated in
    C++/OpenMP (oracle/cpu_kspace.cpp) on the host cores, on the headline's workload.
    Each step is a bounded sample: one k-point per host thread, consecutive points of the
    24 x 24 grid (cycling through it); the line's value is k-points over the summed step
    times.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    from lqm_workloads import lattice as LL
    from lqm_workloads import models as M
    from oracle import cpu as C
    threads = cpu_threads()
    _, h = M.tbg_slater_koster(10)
    ks_all = LL.regulargrid(NK_SIDE * NK_SIDE)
    pk = C._pack(h)
    pos = 0
    for _ in range(args.warmup):
        cpu_density_sample(h, ks_all, pos, threads, threads, pk)
        pos += threads
    t_all = time.perf_counter()
    done, secs = 0, []
    for _ in range(args.steps):
        c, sec = cpu_density_sample(h, ks_all, pos, threads, threads, pk)
        pos += threads
        done += c
        secs.append(sec)
    wall = time.perf_counter() - t_all
    v = done / sum(secs)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "k-pts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(secs) / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded model)",
            "config": {"workload": WORKLOAD, "parallelism": f"dp{world} (k-grid shards)",
                       "host_threads": threads, "k_points_per_step": threads},
            "cpu_baseline": {"value": v, "unit": "k-pts/s", "cores": threads, "kind": "port",
                             "sample": f"per step {threads} consecutive k-points of the 24x24 grid (one per host "
                                       f"thread), C++/OpenMP restatement of the :multithreaded k-loop (H(k), "
                                       f"LAPACK zheevr, zgemm rho_k, fold into the 7 keys), one BLAS thread per "
                                       f"thread; {args.steps} timed steps, wall {wall:.1f} s"},
            "e2e": {"value": v, "unit": "k-pts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ctx_device(ctx):
    return 0 if not hasattr(ctx, "device") else ctx.device


def large_configs(Q, ctx, M, threads):
    """The other configurations of the hot path, one call each after a warm-up call,
    through the host-pointer C-ABI: device time of the call's kernels (CUDA events
    inside the library) and wall time including uploads and result copies."""
    import numpy as np
    from lqm_workloads import lattice as LL
    out = {}

    def timed(fn, reps=1):
        fn()
        best_dev, best_wall = 1e30, 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            best_wall = min(best_wall, time.perf_counter() - t0)
            best_dev = min(best_dev, ctx.last_kernel_ms() / 1e3)
        return best_dev, best_wall

    def density_call(h, ks):
        rho = {R: None for R in h}
        return lambda: Q.getdensitymatrix(rho, h, ks, mu=MU, T=TEMP, ctx=ctx)

    # honeycomb 6x6 spinful with onsite disorder, n = 144, 48 x 48 grid
    _, h1 = M.honeycomb_disorder()
    ks1 = LL.regulargrid(48 * 48)
    dv, wl = timed(lambda: Q.bandmatrix(h1, ks1, ctx=ctx), reps=3)
    dd, wd = timed(density_call(h1, ks1), reps=3)
    out["honeycomb6x6_n144"] = {
        "grid": "48x48", "bands_kpts_per_s": ks1.shape[1] / dv, "bands_wall_kpts_per_s": ks1.shape[1] / wl,
        "rho_kpts_per_s": ks1.shape[1] / dd, "rho_wall_kpts_per_s": ks1.shape[1] / wd,
        "cpu_rho_kpts_per_s": cpu_rate(h1, ks1, threads, per_thread=8),
        "path": "one-CTA-per-k eigensolver, Householder matrix in global scratch (n < 224)"}
    # twisted bilayer m=10, n = 1324: the 400-point k-path (bands only; rho on the 24 x 24
    # grid is the headline)
    lat3, h3 = M.tbg_slater_koster(10)
    kp3 = LL.kpath(lat3, 400)
    db, wb = timed(lambda: Q.bandmatrix(h3, kp3, ctx=ctx))
    out["tbg_m10_n1324_kpath"] = {
        "kpath_points": kp3.shape[1], "kpath_bands_kpts_per_s": kp3.shape[1] / db,
        "kpath_bands_wall_kpts_per_s": kp3.shape[1] / wb,
        "cpu_kpath_bands_kpts_per_s": cpu_rate(h3, kp3, threads, per_thread=2, bands_only=True),
        "path": "batched blocked eigensolver, two-stage reduction (dense -> band of half-bandwidth 16 by panel "
                "QRs and GEMM updates, bulge chase to the tridiagonal), eigenvalue-only merges"}
    # twisted bilayer m=15, n = 2884: one eigen + rho pass over the 12 x 12 grid, then
    # the Hartree-Fock SCF with the screened Coulomb interaction (3 iterations, the
    # 2nd and 3rd replayed from a captured CUDA graph), on a context of its own so that
    # its ~80 GB of work buffers are released afterwards
    ctx5 = Q.Context(ctx_device(ctx), timeout=1800)
    lat5, h5, v5 = M.tbg_screened_hf(15)
    n5 = h5[(0, 0)].shape[0]
    ks5 = LL.regulargrid(12 * 12)
    rho5 = {R: None for R in h5}
    Q.getdensitymatrix(rho5, h5, ks5, mu=MU, T=TEMP, ctx=ctx5)
    t0 = time.perf_counter()
    Q.getdensitymatrix(rho5, h5, ks5, mu=MU, T=TEMP, ctx=ctx5)
    wd = time.perf_counter() - t0
    dd = ctx5.last_kernel_ms() / 1e3
    rng = np.random.default_rng(11)
    X = rng.normal(size=(n5, n5)) * 0.01
    r0 = {R: np.zeros((n5, n5), complex) for R in v5}
    r0[(0, 0)] = 0.5 * np.eye(n5) + (X + X.T)
    iters = 3
    t0 = time.perf_counter()
    res = Q.solvehartreefock(h5, v5, r0, 0.5, ks5, T=0.05, beta=0.3, tol=0.0, iterations=iters, ctx=ctx5)
    t_scf = time.perf_counter() - t0
    out["tbg_m15_n2884"] = {"grid": "12x12", "rho_pass_s": dd, "rho_pass_wall_s": wd,
                            "rho_kpts_per_s": ks5.shape[1] / dd, "path": "batched blocked eigensolver",
                            "scf": {"interaction": "screened Coulomb V0 e^{-r/lam}/r, V0 = 1.4 eV a, lam = 10 a, "
                                                   "onsite 1.4 eV, 9 keys", "iterations": iters,
                                    "s_per_iter": t_scf / iters,
                                    "device_s_per_iter": ctx5.last_kernel_ms() / 1e3 / iters,
                                    "residual": res.residual,
                                    "note": "wall time of lqm_scf_hf incl. the first (uncaptured) iteration "
                                            "and the h/v/rho uploads"},
                            "cpu": "not sampled (about a minute per k-point and core)"}
    ctx5.close()
    # adjoint: density-response VJP on the triangular Hubbard model (n = 72, 36 x 36)
    _, h4, _ = M.triangular_hubbard(L_super=6)
    ks4 = LL.regulargrid(36 * 36)
    n4 = h4[(0, 0)].shape[0]
    rng = np.random.default_rng(1)
    G = {(0, 0): rng.normal(size=(n4, n4)) + 1j * rng.normal(size=(n4, n4))}
    dv, wv = timed(lambda: Q.densitymatrix_vjp(h4, ks4, G, mu=0.0, T=0.02, ctx=ctx), reps=3)
    out["vjp_triangular_n72"] = {"grid": "36x36", "vjp_kpts_per_s": ks4.shape[1] / dv,
                                 "vjp_wall_kpts_per_s": ks4.shape[1] / wv}
    # Kubo correlator chi_xx(w) and chi_xy(w) (64 frequencies, Gamma = 0.05, T = 0.01) on the
    # honeycomb 6x6 cell (48 x 48 grid) and the m=10 twisted bilayer (8 x 8 grid)
    om = np.linspace(0.0, 3.0, 64)
    kubo = {}
    for name, lat, h, ks in (("honeycomb6x6_n144", *M.honeycomb_disorder(), ks1),
                             ("tbg_m10_n1324", lat3, h3, LL.regulargrid(8 * 8))):
        J = M.currentoperators(lat, h)
        Hd, J0, J1 = Q.DeviceHops(h, ctx), Q.DeviceHops(J[0], ctx), Q.DeviceHops(J[1], ctx)
        dxx, wxx = timed(lambda: Q.opticalconductivity(om, Hd, J0, J0, ks, Gamma=0.05, T=0.01, ctx=ctx))
        dxy, wxy = timed(lambda: Q.opticalconductivity(om, Hd, J0, J1, ks, Gamma=0.05, T=0.01, ctx=ctx))
        dbv, _ = timed(lambda: Q.bandmatrix(Hd, ks, want_vectors=True, ctx=ctx))
        kubo[name] = {"kpoints": ks.shape[1], "frequencies": len(om),
                      "xx_kpts_per_s": ks.shape[1] / dxx, "xx_wall_kpts_per_s": ks.shape[1] / wxx,
                      "xy_kpts_per_s": ks.shape[1] / dxy, "xy_wall_kpts_per_s": ks.shape[1] / wxy,
                      "eigen_pass_with_vectors_kpts_per_s": ks.shape[1] / dbv}
    out["optical_conductivity"] = kubo
    return out


def measured_fp64_peak(torch, dev):
    """cuBLAS DGEMM (8192^3) best of 5, TFLOP/s; the FP64 denominator of the pass's
    flop rate (MEASURED_PEAKS.json carries no FP64 figure)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2 * 8192 ** 3 / best / 1e12


def profile_case(Q, ctx, h, torch, dev, np):
    """A small case of the bench's dominant kernel for profilers: 2048 k-points of the
    n=96 model through lqm_bands_dos_rho_dev (one eigh_kernel launch)."""
    nk = 2048
    ks = np.random.default_rng(0).random((2, nk))
    d_ks = torch.from_numpy(np.ascontiguousarray(ks.T)).to(dev)
    Hd = Q.DeviceHops(h, ctx)
    n = Hd.n
    Lk = np.asfortranarray(np.array(list(h.keys()), dtype=np.int64).T)
    rho = torch.zeros(len(h), n, n, dtype=torch.complex128, device=dev)
    bands = torch.zeros(nk, n, dtype=torch.float64, device=dev)
    dos = torch.zeros(NW, dtype=torch.float64, device=dev)
    om = torch.linspace(-6.0, 6.0, NW, dtype=torch.float64, device=dev)
    eb = ctypes.c_double()
    for _ in range(2):
        ctx.check(Q.lib().lqm_bands_dos_rho_dev(ctx.handle, Hd.handle, nk, Q._ptr(d_ks), None, MU, TEMP, len(h),
                                                 Q._ptr(Lk), Q._ptr(rho), ctypes.byref(eb), NW, Q._ptr(om), GAMMA,
                                                 Q._ptr(dos), Q._ptr(bands), 0))
    print(json.dumps({"profile_case": "n=96 batch model, 2048 k", "kernel_ms": ctx.last_kernel_ms()}))


def profile_case_tbg(Q, ctx, M, case):
    """Small cases of the blocked path for profilers: one call on the twisted
    bilayer m=10 (n=1324) over the first nk points of the 24x24 grid."""
    from lqm_workloads import lattice as LL
    kind = "bands" if case.startswith("tbg10-bands") else "density"
    nk = int(case.rsplit("bands", 1)[-1]) if kind == "bands" else int(case.rsplit("density", 1)[-1])
    _, h = M.tbg_slater_koster(10)
    ks = LL.regulargrid(24 * 24)[:, :nk]
    t0 = time.perf_counter()
    if kind == "bands":
        Q.bandmatrix(h, ks, ctx=ctx)
    else:
        rho = {R: None for R in h}
        Q.getdensitymatrix(rho, h, ks, mu=MU, T=TEMP, ctx=ctx)
    print(json.dumps({"profile_case": case, "kernel_ms": ctx.last_kernel_ms(), "wall_s": time.perf_counter() - t0}))


def profile_case_kubo(Q, ctx, M):
    """One Kubo correlator call for profilers: chi_xy(w) of the disordered honeycomb 6x6
    cell (n = 144) over the 48 x 48 grid, 64 frequencies."""
    import numpy as np
    from lqm_workloads import lattice as LL
    lat, h = M.honeycomb_disorder()
    J = M.currentoperators(lat, h)
    ks = LL.regulargrid(48 * 48)
    t0 = time.perf_counter()
    Q.opticalconductivity(np.linspace(0.0, 3.0, 64), h, J[0], J[1], ks, Gamma=0.05, T=0.01, ctx=ctx)
    print(json.dumps({"profile_case": "kubo144", "kernel_ms": ctx.last_kernel_ms(),
                      "wall_s": time.perf_counter() - t0}))


def batch_config(Q, ctx, M, torch, dev, np, steps, fp64_peak):
    """The batched three-model configuration (n = 8, 24, 96; 256 x 256 k each): bands +
    DOS + rho_R through lqm_bands_dos_rho_dev with device-resident inputs, 3 warm-up
    steps and `steps` timed steps; the one-CTA eigensolver's FP64 roofline per model."""
    models = M.batch_models()
    ks_np = kgrid(0, 1)
    nk = ks_np.shape[1]
    d_ks = torch.from_numpy(np.ascontiguousarray(ks_np.T)).to(dev)
    state = []
    for name, h in models:
        Hd = Q.DeviceHops(h, ctx)
        n = Hd.n
        Lk = np.asfortranarray(np.array(list(h.keys()), dtype=np.int64).T)
        d_bands = torch.zeros(nk, n, dtype=torch.float64, device=dev)
        ctx.check(Q.lib().lqm_bandmatrix_dev(ctx.handle, Hd.handle, nk, Q._ptr(d_ks), 0, 0, Q._ptr(d_bands), None))
        lo, hi = float(d_bands.min()), float(d_bands.max())
        state.append(dict(name=name, Hd=Hd, n=n, nR=len(h), Lk=Lk, bands=d_bands,
                          rho=torch.zeros(len(h), n, n, dtype=torch.complex128, device=dev),
                          dos=torch.zeros(NW, dtype=torch.float64, device=dev),
                          om=torch.linspace(lo, hi, NW, dtype=torch.float64, device=dev)))
    block_sizes = {}
    for s_ in state:
        if s_["n"] < 128:
            best, _, table = Q.autotune_eigh(s_["Hd"], ks_np, want_rho=True, ctx=ctx)
            block_sizes[f"n{s_['n']}"] = best
    eb = ctypes.c_double()

    def step(per_model_ms=None):
        for s_ in state:
            m0 = ctx.stats()[0]
            ctx.check(Q.lib().lqm_bands_dos_rho_dev(
                ctx.handle, s_["Hd"].handle, nk, Q._ptr(d_ks), None, MU, TEMP, s_["nR"], Q._ptr(s_["Lk"]),
                Q._ptr(s_["rho"]), ctypes.byref(eb), NW, Q._ptr(s_["om"]), GAMMA, Q._ptr(s_["dos"]),
                Q._ptr(s_["bands"]), 0))
            if per_model_ms is not None:
                per_model_ms[s_["n"]] = per_model_ms.get(s_["n"], 0.0) + ctx.stats()[0] - m0

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    ctx.reset_stats(timing=True)
    per_model_ms = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step(per_model_ms)
    e1.record()
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    ctx.stats()  # collects the pending events
    detail = {}
    for s_ in state:
        ms = per_model_ms.get(s_["n"], 0.0)
        tf = steps * nk * eigh_flops_per_k(s_["n"], s_["nR"]) / (ms / 1e3) / 1e12 if ms > 0 else None
        detail[f"n{s_['n']}"] = {"eigh_ms_per_step": ms / steps, "eigh_tflops": tf,
                                 "eigh_frac_of_fp64": (tf / fp64_peak) if tf else None,
                                 "eigh_block_size": block_sizes.get(f"n{s_['n']}")}
    # the same step with ONE eigensolver launch for the three models (sub-teams per CTA)
    multi = [dict(H=s_["Hd"], Lk=s_["Lk"], rho=s_["rho"], om=s_["om"], dos=s_["dos"], bands=s_["bands"])
             for s_ in state]
    for _ in range(3):
        Q.bands_dos_rho_multi_dev(multi, d_ks, nk, mu=MU, T=TEMP, gamma=GAMMA, ctx=ctx)
    torch.cuda.synchronize()
    ctx.reset_stats(timing=True)
    e0.record()
    for _ in range(steps):
        Q.bands_dos_rho_multi_dev(multi, d_ks, nk, mu=MU, T=TEMP, gamma=GAMMA, ctx=ctx)
    e1.record()
    torch.cuda.synchronize()
    el1 = e0.elapsed_time(e1) / 1e3
    eigh_ms1, eigh_launches1, _ = ctx.stats()
    for s_ in state:
        s_["Hd"].free()
    return {"workload": BATCH_WORKLOAD, "kpts_per_s": len(state) * nk * steps / el, "ms_per_step": 1000 * el / steps,
            "steps": steps, "warmup": 3, "per_model": detail,
            "eigh_flops_per_k": "8 nR n^2 + 13.33 n^3 (Bloch sum + eigh with vectors; rho_k fused, not counted)",
            "one_launch": {"kpts_per_s": len(state) * nk * steps / el1, "ms_per_step": 1000 * el1 / steps,
                           "eigh_launches_per_step": eigh_launches1 / steps, "eigh_ms_per_step": eigh_ms1 / steps,
                           "note": "lqm_bands_dos_rho_multi_dev: the three models' k-points in one eigensolver "
                                   "launch (CTA sub-teams of each model's block size), then the per-model folds "
                                   "and DOS"}}


def main():
    # the SCF timings run a fixed number of iterations (tol = 0): no convergence warnings
    warnings.filterwarnings("ignore", message="SCF stopped before reaching the tolerance")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (batch of n=8/24/96, n=144, the k-path, n=2884, SCF, "
                         "the adjoint, Kubo)")
    ap.add_argument("--profile-case", nargs="?", const="n96", default=None,
                    choices=["n96", "tbg10-bands576", "tbg10-bands16", "tbg10-density142", "tbg10-density16", "kubo144"],
                    help="one call of a small profiling case: n96 = the fused bench call on the n=96 model "
                         "over 2048 k; tbg10-* = bands or density of the n=1324 twisted bilayer over the "
                         "first 576 / 142 / 16 points of the 24x24 grid; kubo144 = the Kubo correlator "
                         "of the n=144 honeycomb cell over 48x48 k and 64 frequencies")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.warmup < 3:
        args.warmup = 3

    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "latticeqm.jl_b200"))
    import build as lqm_build
    if not os.path.exists(lqm_build.LIB):
        lqm_build.build()
    import lqm_cuda as Q
    from lqm_workloads import lattice as LL
    from lqm_workloads import models as M

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ctx = Q.Context(local, timeout=900)
    if args.profile_case == "n96":
        return profile_case(Q, ctx, M.batch_models()[2][1], torch, dev, np)
    if args.profile_case == "kubo144":
        return profile_case_kubo(Q, ctx, M)
    if args.profile_case:
        return profile_case_tbg(Q, ctx, M, args.profile_case)

    # ---- the library's communicator: k-point shards, rho_L summed over the ranks ----
    if world > 1:
        uid = Q.comm_unique_id() if rank == 0 else None
        box = [uid]
        dist.broadcast_object_list(box, src=0)
        ctx.set_comm(world, rank, box[0])

    # ---- device-resident inputs ----
    _, h = M.tbg_slater_koster(10)
    keys = list(h.keys())
    ks_np = full_grid(world)
    nk = ks_np.shape[1]
    nk_local = nk // world
    d_ks = torch.from_numpy(np.ascontiguousarray(ks_np.T)).to(dev)   # (nk, 2) row-major == (2, nk) col-major
    Hd = Q.DeviceHops(h, ctx)
    n, nR = Hd.n, Hd.nR
    Lk = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    # the reduction (one- or two-stage) measured on half of this model's grid before the
    # warm-up (one GPU; with several, every rank keeps the library's default)
    reduction = {"choice": "two-stage (library default for density passes)"}
    if world == 1:
        best_r, _, table_r = Q.autotune_eigh(Hd, ks_np[:, :288], want_rho=True, ctx=ctx)
        reduction = {"choice": "two-stage" if best_r == 1 else "one-stage", "autotuned": True,
                     "pass_ms": {("two-stage" if k == 1 else "one-stage"): v for k, v in table_r.items()}}
    d_rho = torch.zeros(nR, n, n, dtype=torch.complex128, device=dev)
    eb = ctypes.c_double()

    def step():
        ctx.check(Q.lib().lqm_densitymatrix_dev(ctx.handle, Hd.handle, nk, Q._ptr(d_ks), None, MU, TEMP, nR,
                                                Q._ptr(Lk), Q._ptr(d_rho), ctypes.byref(eb), 0))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region (device resident) ----
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ctx.reset_stats(timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    elapsed = e0.elapsed_time(e1) / 1e3
    clocks = sampler.stop()
    eigh_ms, eigh_launches, launches = ctx.stats()
    symv_ms, symv_launches, symv_bytes = ctx.kernel_stats(1)
    q2_ms, q2_launches, q2_flops = ctx.kernel_stats(2)
    if world > 1:
        t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t[0])
    total_k = nk * args.steps
    value = total_k / elapsed

    # ---- e2e through the host-pointer C-ABI from pinned host memory ----
    _, _, d_, K_, B_ = Q.pack_hops(h)
    blocks_pin = torch.from_numpy(np.ascontiguousarray(B_.transpose(2, 1, 0))).pin_memory()  # n x n x nR col-major
    keys_pin = torch.from_numpy(np.ascontiguousarray(K_.T)).pin_memory()
    ks_pin = torch.from_numpy(np.ascontiguousarray(ks_np.T)).pin_memory()
    rho_pin = torch.zeros(nR, n, n, dtype=torch.complex128).pin_memory()
    h2d = blocks_pin.numel() * 16 + keys_pin.numel() * 8 + ks_pin.numel() * 8
    d2h = rho_pin.numel() * 16 + 8

    def e2e_step():
        hp = ctypes.c_void_p()
        ctx.check(Q.lib().lqm_hops_upload_dense(ctx.handle, n, nR, d_, Q._ptr(keys_pin), Q._ptr(blocks_pin),
                                                ctypes.byref(hp)))
        ctx.check(Q.lib().lqm_densitymatrix(ctx.handle, hp, nk, Q._ptr(ks_pin), None, MU, TEMP, nR, Q._ptr(Lk),
                                            Q._ptr(rho_pin), ctypes.byref(eb), 0))
        ctx.check(Q.lib().lqm_hops_free(ctx.handle, hp))

    e2e_steps = max(3, args.steps // 4)
    e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_el = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_el], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_el = float(t[0])
    e2e_val = nk * e2e_steps / e2e_el

    # ---- roofline of the dominant kernel ----
    # two-stage reduction (the default on the blocked path): the stage-2
    # back-transformation, FP64-bound, against the FP64 GEMM rate measured in this run;
    # one-stage (LQM_TWO_STAGE=0): the lower-triangle mat-vec, HBM-bound
    fl = flops_per_k(n, nR, nR)
    fp64_peak = measured_fp64_peak(torch, dev)
    if q2_launches:
        achieved = q2_flops / (q2_ms / 1e3) / 1e12 if q2_ms > 0 else None
        per_launch = q2_flops / q2_launches
        traffic = None
        tfile = os.path.join(ROOT, "profiles", "q2g_traffic.json")
        if os.path.exists(tfile):
            try:
                traffic = json.load(open(tfile))["dram_bytes_per_algorithmic_flop"] * per_launch
            except Exception:
                traffic = None
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": (achieved / fp64_peak) if achieved else None, "traffic": traffic,
                "kernel": "ts_q2g_kernel (two-stage reduction: the bulge-chasing reflectors applied to the needed "
                          "eigenvector columns in groups of 16 sweeps, a 31-row register window per column; "
                          "one launch per batch)",
                "algorithmic_flops_per_launch": per_launch,
                "algorithmic_flops_per_k": "8 n (n-1) per eigenvector column formed (each reflector row: dot and "
                                           "update, 8 real flops each; the columns that carry rho_k)",
                "launches": q2_launches, "kernel_ms": q2_ms, "share_of_step": q2_ms / 1e3 / elapsed,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64; MEASURED_PEAKS.json has no FP64 "
                               "figure); the kernel runs on the FP64 FMA pipe, whose rate matches the FP64 tensor "
                               "rate on B200",
                "traffic_source": "ncu dram bytes / algorithmic flops of one capture (profiles/q2g_traffic.json) "
                                  "x this run's algorithmic flops per launch",
                "pass_tflops": value / world * fl / 1e12, "pass_flops_per_k": fl,
                "eigh_pass_ms": eigh_ms, "eigh_passes": eigh_launches}
    else:
        peak, peak_src = hbm_peak()
        achieved = symv_bytes / (symv_ms / 1e3) / 1e9 if symv_ms > 0 else None
        per_launch = symv_bytes / symv_launches if symv_launches else None
        traffic = None
        tfile = os.path.join(ROOT, "profiles", "blk_symv_traffic.json")
        if per_launch and os.path.exists(tfile):
            try:
                traffic = json.load(open(tfile))["dram_bytes_per_algorithmic_byte"] * per_launch
            except Exception:
                traffic = None
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": "blk_symv_tma_kernel (Householder mat-vec y = A22 v over the lower triangle of the "
                          "trailing block, 64x64 tiles moved by TMA, all k-points of the batch per launch; one "
                          "launch per column)",
                "algorithmic_bytes_per_launch": per_launch,
                "algorithmic_bytes_per_k": "16 B x m(m+1)/2 per column, m = n-1-j (sum ~ 16 n^3/6 = 6.2 GB at n=1324)",
                "launches": symv_launches, "kernel_ms": symv_ms, "share_of_step": symv_ms / 1e3 / elapsed,
                "peak_source": peak_src,
                "traffic_source": "ncu dram bytes / algorithmic bytes of one capture (profiles/blk_symv_traffic.json) "
                                  "x this run's algorithmic bytes per launch",
                "pass_tflops": value / world * fl / 1e12, "pass_flops_per_k": fl,
                "eigh_pass_ms": eigh_ms, "eigh_passes": eigh_launches}
    roof["fp64_dgemm_tflops_measured"] = fp64_peak
    roof["pass_frac_of_fp64"] = roof["pass_tflops"] / fp64_peak

    threads = cpu_threads()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_tbg(h, LL.regulargrid(NK_SIDE * NK_SIDE), threads)

    configs = None
    scf = None
    if rank == 0 and world == 1 and not args.no_configs:
        Hd.free()
        del d_rho
        torch.cuda.empty_cache()
        configs = {"batch3": batch_config(Q, ctx, M, torch, dev, np, 3, fp64_peak)}
        lat4, h4, v4 = M.triangular_hubbard(L_super=6)
        rho0 = {(0, 0): M.random_local_magnetization(lat4.norb, seed=3)}
        ks4 = LL.regulargrid(36 * 36)
        Q.solvehartreefock(h4, v4, rho0, 0.5, ks4, T=0.02, beta=0.3, tol=0.0, iterations=3, ctx=ctx)
        iters = 12
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = Q.solvehartreefock(h4, v4, rho0, 0.5, ks4, T=0.02, beta=0.3, tol=0.0, iterations=iters, ctx=ctx)
        t_scf = time.perf_counter() - t0
        scf = {"workload": "triangular 6x6 spinful Hubbard HF (n=72, U=4, t'=0.2), 36x36 k, T=0.02, beta=0.3",
               "s_per_iter": t_scf / iters, "device_ms_per_iter": ctx.last_kernel_ms() / iters,
               "iterations": iters, "residual": res.residual,
               "note": "wall time of lqm_scf_hf per iteration incl. h/v upload and the returned rho; "
                       "iterations 2+ replay a captured CUDA graph"}
        configs.update(large_configs(Q, ctx, M, threads))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "k-pts/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded model)",
                "config": {"workload": WORKLOAD, "k_points_per_gpu_per_step": nk_local, "reduction": reduction,
                           "parallelism": f"dp{world} (k-grid shards in the library; rho_R all-reduce over NCCL)"
                           if world > 1 else "dp1",
                           "l2": "inputs larger than L2 (each step streams ~32 GB of A/U through HBM)",
                           "precision": "FP64 plain (the mixed-precision form is not built)"},
                "e2e": {"value": e2e_val, "unit": "k-pts/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "steps": e2e_steps},
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks, "scf": scf,
                "configs": configs}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
