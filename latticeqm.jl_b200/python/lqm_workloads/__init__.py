"""Seeded synthetic inputs for the k-space hot path, in LatticeQM's Hops format.

The reference builds its tight-binding models on the host in Julia
(src/modules/Structure, src/modules/Operators); that construction is not part
of the accelerated path.  This package restates the pieces needed to produce
the named workloads (lattices, supercells, twisted bilayers, hopping rules,
Hubbard interaction, seeded disorder) so the CUDA path can be driven and
benchmarked without Julia.  `lattice` holds the geometry, `models` the Hops
builders.  Pure NumPy; no dependency on the CUDA library.
"""
