"""The accuracy bar of the eigen pass against single precision, on the twisted bilayer.

The band accuracy asked of any faster variant is 1e-8 of the spectral width (the
FP64 LAPACK `zheevr` call of src/modules/Eigen/Eigen.jl:22-23 being the reference).
This study fixes two facts the library's choice of an FP64 pipeline rests on, with
LAPACK on the host (numpy) and the model of the n = 1324 headline configuration:

* an eigensolve carried out wholly in single precision misses that bar (its band
  error is a few 1e-8 of the width at n = 1324);
* its eigenvectors, refined by one FP64 Rayleigh quotient (H U and the column dot
  products: 8 n^3 flops of FP64 GEMM per k-point), meet it by orders of magnitude.

So a mixed form needs FP64 work of at least 8 n^3 per k-point on top of the
single-precision solve, more than the FP64 eigenvalue-only two-stage reduction's
16/3 n^3.  Host-only (no device); one k-point, a few seconds.
"""
import numpy as np
import pytest

from oracle import kspace as K
from lqm_workloads import models as M

BAR = 1e-8


@pytest.fixture(scope="module")
def tbg_hk():
    _, h = M.tbg_slater_koster(10)
    return K.fouriersum(h, np.array([0.13, 0.37]))


def test_single_precision_eigensolve_misses_the_band_bar(tbg_hk):
    H = tbg_hk
    assert H.shape == (1324, 1324)
    e64 = np.linalg.eigvalsh(H)
    e32 = np.linalg.eigvalsh(H.astype(np.complex64)).astype(np.float64)
    width = e64[-1] - e64[0]
    err = np.abs(e32 - e64).max() / width
    assert err > BAR, err
    assert err < 1e-6, err


def test_fp64_rayleigh_quotient_of_single_precision_vectors_meets_it(tbg_hk):
    H = tbg_hk
    e64 = np.linalg.eigvalsh(H)
    _, U32 = np.linalg.eigh(H.astype(np.complex64))
    U = U32.astype(np.complex128)
    rq = np.real(np.einsum("ij,ij->j", U.conj(), H @ U)) / np.real(np.einsum("ij,ij->j", U.conj(), U))
    width = e64[-1] - e64[0]
    err = np.abs(np.sort(rq) - e64).max() / width
    assert err < 1e-3 * BAR, err
