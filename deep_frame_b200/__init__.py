"""B200 (sm_100a) implementation of the hex8 SIMP topology-optimisation hot path.

The compute runs in ``libtfb200.so`` (hand-written CUDA behind the C ABI of
``include/tf_b200.h``); this package holds the host-side mirror of the
reference interfaces that sit on that path.
"""
from .elements import _CORNERS, elasticity_matrix, hexahedron_matrices, orthotropic_matrix, regular_grid, select_nodes, simp

__all__ = ["_CORNERS", "elasticity_matrix", "hexahedron_matrices", "orthotropic_matrix", "regular_grid", "select_nodes", "simp"]
