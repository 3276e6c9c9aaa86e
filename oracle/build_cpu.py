"""Build the oracle's C++/OpenMP restatement (oracle/cpu_kspace.cpp) into
oracle/lib/libcpu_kspace.so.  Test infrastructure: the checker and the timed CPU
baseline only.

It links the zheevr/zgemm of the OpenBLAS that SciPy ships (scipy.libs), found
next to the installed scipy package; the image is the same here and on the GPU
hosts, so the built library travels with the repository.

    python oracle/build_cpu.py
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_kspace.cpp")
LIB = os.path.join(HERE, "lib", "libcpu_kspace.so")


def scipy_openblas():
    import scipy
    libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libs, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError(f"no libscipy_openblas*.so under {libs}")
    return cands[0]


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    blas = scipy_openblas()
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fopenmp", "-shared", "-fPIC", SRC,
           "-L" + os.path.dirname(blas), "-l:" + os.path.basename(blas),
           "-Wl,-rpath," + os.path.dirname(blas), "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
