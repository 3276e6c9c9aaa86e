"""Build libkspace.so (sm_100a) in-tree with nvcc.

Usage: python latticeqm.jl_b200/build.py [--force]
Output: latticeqm.jl_b200/lib/libkspace.so
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libkspace.so")
SOURCES = ["lqm_capi.cu"]
DEPS = ["lqm_capi.cu", "lqm_kernels.cuh", "lqm_eigh.cuh", "lqm_team.cuh", "lqm_hf.cuh", "lqm_scf.inc", "lqm_plan.h",
        "lqm_blocked.cuh", "lqm_large.cuh", "lqm_adjoint.inc", "lqm_obs.inc", "lqm_anderson.inc",
        "lqm_sitedos.inc", "lqm_berry.inc", "lqm_kubo.inc", "lqm_partial.inc", "lqm_commutator.inc", "lqm_bdg.inc", "lqm_scf_bdg.inc", "lqm_autotune.inc", "lqm_comm.inc", "lqm_scfgrad.inc", "lqm_zgemm.cuh", "lqm_twostage.cuh"]
CUDA_LIB = "/usr/local/cuda/lib64"
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    srcs = [os.path.join(CSRC, f) for f in DEPS] + [os.path.join(ROOT, "include", "kspace.h")]
    return all(os.path.getmtime(s) <= t for s in srcs)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
           *[os.path.join(CSRC, s) for s in SOURCES], "-L", CUDA_LIB,
           "-Xlinker", "-rpath=" + CUDA_LIB, "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
