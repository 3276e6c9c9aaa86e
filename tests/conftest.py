import os
import sys

# The oracle makes many small LAPACK calls (n <= 144 per k-point); a multi-threaded
# BLAS spends most of their time synchronising its threads (84 s against 2.6 s for
# one SCF iteration of the n = 72, 36 x 36 model on 8 cores), so it runs on one.
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "latticeqm.jl_b200")
for p in (ROOT, os.path.join(PKG, "python")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path via the C-ABI")


@pytest.fixture(scope="session")
def lqm():
    """The ctypes mirror of the C-ABI, with the library built in-tree."""
    sys.path.insert(0, PKG)
    import build as _build  # latticeqm.jl_b200/build.py
    _build.build()
    import lqm_cuda
    return lqm_cuda


@pytest.fixture(scope="session")
def ctx(lqm):
    c = lqm.Context(0, timeout=600)
    yield c
    c.close()
