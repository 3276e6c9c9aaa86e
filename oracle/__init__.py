"""CPU oracle for the LatticeQM k-space hot path.

TEST INFRASTRUCTURE ONLY.  This package restates, in NumPy/SciPy, the
reference algorithms of LatticeQM.jl (pure Julia) that the CUDA library
replaces: the Bloch sum, the dense Hermitian eigensolve (LAPACK ``zheevr`` on the upper
triangle, via SciPy's ``driver='evr'``), the Fermi-Dirac occupation, the
chemical-potential search, the density-matrix fold, the DOS and the
Hartree-Fock self-consistent loop.  Each function cites the reference
``file:line`` it follows.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this package, and only
as the checker or as the timed CPU baseline.  The product path
(``latticeqm.jl_b200``) never imports it.

Inputs come from ``latticeqm.jl_b200/python/lqm_workloads`` (the seeded model
builders shared by the tests and the benchmark).

Pinning: the restatement is checked against the reference's own golden
vectors (analytic graphene/square/triangular bands, twisted-bilayer
eigenvalue fixtures, DOS sum rules, the HF variational identity); see
``tests/test_oracle_pins.py``.
"""
