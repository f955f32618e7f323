"""Batched problems: the k-points of one cell and an ensemble of strained cells.

The reference solves every (spin, k-point) of a cell one after another
(SCF::solve_eigenproblem, src/scf/SCF.cpp:383-410, each a call of EigenSolver::solve_kpt);
an ensemble of cells is a loop of independent SCF runs.  Each such problem here is a
`Problem` (its own grid, k-point, projectors, potential and band count), and
`lynx_b200.solver.solve_batch` runs one CheFSI pass over a list of them at once.

`kpoint_problems` and `strained_ensemble` build seeded synthetic inputs for the two kinds:
the primitive FCC Si cell on a Monkhorst-Pack grid (complex Bloch orbitals) and conventional
Si8 cells with isotropic strain and grids drawn from a list.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import cell as C
from . import pseudo as P


@dataclass
class Problem:
    cell: C.Cell
    positions: np.ndarray
    veff: np.ndarray
    nband: int
    kcart: Optional[np.ndarray] = None  # None: Gamma point, real orbitals
    weight: float = 1.0
    tables: Optional[P.NonlocalTables] = None

    @property
    def complex(self) -> bool:
        return self.kcart is not None


def kpoint_problems(psp: P.Psp8, kgrid: Sequence[int] = (4, 4, 4), grid: int = 20, nband: int = 16,
                    seed: int = 0) -> List[Problem]:
    """Primitive FCC Si (2 atoms) at every reduced Monkhorst-Pack k-point (time-reversal
    pairs merged, weight 2), complex orbitals.  The k-points share the cell, the potential
    and the projector tables."""
    cl, pos = C.fcc_si_primitive(grid)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=seed)
    tab = P.nonlocal_tables(cl, pos, psp)
    kc, _, w = C.kpoints_mp(cl, kgrid)
    return [Problem(cl, pos, V, nband, kc[i].copy(), float(w[i]), tab) for i in range(len(kc))]


def strained_ensemble(psp: P.Psp8, n_cells: int = 32, grids: Sequence[int] = (24, 26, 28, 30, 32),
                      max_strain: float = 0.03, nband: int = 24, seed: int = 0) -> List[Problem]:
    """Si8 conventional cells with seeded isotropic strain uniform(-max_strain, max_strain) and
    grids drawn uniformly from `grids` (per axis the same), Gamma point."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_cells):
        eps = float(rng.uniform(-max_strain, max_strain))
        g = int(rng.choice(np.asarray(grids)))
        cl, pos = C.diamond_si(1, g, strain=eps, seed=seed + i)
        V = C.synthetic_veff(cl, pos, noise=1e-3, seed=seed + i)
        out.append(Problem(cl, pos, V, nband, None, 1.0, P.nonlocal_tables(cl, pos, psp)))
    return out
