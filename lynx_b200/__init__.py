"""lynx_b200: B200-native CheFSI eigensolver hot path of the LYNX real-space DFT code.

The operators run in liblynxb200.so (hand-written sm_100a CUDA behind the C ABI in
include/lynx_b200.h); this package holds the host-side set-up (cell geometry, k-points,
pseudopotential projector tables) and the Python mirror of the reference operator API.
"""
from . import cell, pseudo
from .cell import Cell, diamond_si, fcc_si_primitive, kpoints_mp, random_orbitals, synthetic_veff
from .pseudo import NonlocalTables, nonlocal_tables, read_psp8, synthetic_si_psp8

__all__ = [
    "cell", "pseudo", "Cell", "diamond_si", "fcc_si_primitive", "kpoints_mp", "random_orbitals",
    "synthetic_veff", "NonlocalTables", "nonlocal_tables", "read_psp8", "synthetic_si_psp8",
    "Context", "Hamiltonian", "EigenSolver", "NonlocalProjector", "fermi_level", "occupations",
    "solve_batch",
]


def __getattr__(name):
    # The operator classes load liblynxb200.so on first use.
    if name in ("Context", "Hamiltonian", "EigenSolver", "NonlocalProjector", "fermi_level", "occupations",
                "solve_batch"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
