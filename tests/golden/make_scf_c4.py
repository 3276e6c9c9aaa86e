"""Generate the oracle's converged Hartree-Fock SCF of the triangular Hubbard model
at its full size (n = 72, 36 x 36 k-grid) as a fixture for the GPU parity test.

Model: triangular-lattice Hubbard, 6 x 6 supercell, spinful (n = 72), NN t = -1,
NNN t' = 0.2, U = 4 in the sigma_x mode; seeded random local magnetisation
(seed 7) as the initial density; T = 0.02, filling 0.5, linear mixing
beta = 0.3, stopped at the relative residual 1e-9 (the reference's
_scf_driver!/fixedpoint!, restated in oracle/meanfield.py).

The oracle's SCF loop (oracle/meanfield.py) runs with its k-loops (eigenvalues
for mu, then the density matrix) computed by the oracle's C++/OpenMP
restatement (oracle/cpu.py, the same per-k zheevr, rho_k and fold; pinned to the
Python k-loop in tests/test_oracle_pins.py), ~0.4 s per iteration on 8 cores
instead of ~3 s; the run is done once here and its result committed:

    OPENBLAS_NUM_THREADS=1 python tests/golden/make_scf_c4.py

writes tests/golden/scf_c4_oracle.npz (rho at the zero key, E, mu, residual,
iterations, converged, and the energies eband/eH/eF).
"""
import os
import sys
import time

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "latticeqm.jl_b200", "python")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

from lqm_workloads import lattice as L  # noqa: E402
from lqm_workloads import models as M  # noqa: E402
from oracle import meanfield as MF  # noqa: E402

OUT = os.path.join(HERE, "scf_c4_oracle.npz")
PARAMS = dict(L_super=6, seed=7, nk_side=36, T=0.02, filling=0.5, beta=0.3, tol=1e-9, maxiter=600)


def main():
    p = PARAMS
    lat, h, v = M.triangular_hubbard(L_super=p["L_super"])
    rho0 = {(0, 0): M.random_local_magnetization(lat.norb, seed=p["seed"])}
    ks = L.regulargrid(p["nk_side"] ** 2)
    t0 = time.time()

    def log(it, E, res, *rest):
        print(f"iter {it:4d}  E {E:.15f}  residual {res:.3e}  ({time.time() - t0:.0f} s)", flush=True)

    from oracle import cpu as C
    from oracle import kspace as K
    K.bandmatrix = lambda hh, kk, vectors=False: (C.bandmatrix(hh, kk), None)
    K.densitymatrix = lambda hh, kk, w, mu, T, Lk, return_parts=False: C.densitymatrix(hh, kk, w, mu, T, Lk)
    rho, E, hf, conv, resid, it = MF.solvehartreefock(h, v, rho0, p["filling"], ks, T=p["T"], beta=p["beta"],
                                                      tol=p["tol"], iterations=p["maxiter"], log=log)
    np.savez_compressed(OUT, rho0=rho[(0, 0)], E=E, mu=hf.mu, residual=resid, iterations=it, converged=conv,
                        eband=hf.eband, eH=hf.eH, eF=hf.eF, **{k: v for k, v in p.items()})
    print(f"wrote {OUT}: converged={conv} iterations={it} residual={resid:.3e} E={E:.15f} mu={hf.mu:.15f}")


if __name__ == "__main__":
    main()
