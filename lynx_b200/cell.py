"""Cell geometry, k-points and the synthetic silicon workloads (host side, FP64).

* ``Cell``            — lattice + FD grid: spacing L_i/N_i (periodic) or L_i/(N_i-1)
                        (Dirichlet), dV = |det A| / prod(intervals), unit lattice vectors
                        and lapc_T (src/core/FDGrid.cpp:8-37, src/core/Lattice.cpp:13-51).
* ``kpoints_mp``      — Monkhorst-Pack grid with time-reversal reduction in the
                        reference's folding convention (src/core/KPoints.cpp:8-80).
* ``diamond_si``      — Si diamond cells and supercells (a = 10.26 Bohr) and the
                        primitive FCC cell, with seeded displacements / strain.
* ``synthetic_veff``  — a smooth V_eff (sum of Gaussian wells on the atoms plus seeded
                        noise) standing in for a converged Kohn-Sham potential.
* ``random_orbitals`` — seeded U(-0.5, 0.5) initial orbitals (Wavefunction::randomize
                        convention, src/electronic/Wavefunction.cpp:53-63; numpy's
                        generator replaces std::rand).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Sequence, Tuple

import numpy as np

SI_A = 10.26  # Bohr


@dataclasses.dataclass
class Cell:
    latvec: np.ndarray          # 3x3, rows are lattice vectors (Bohr)
    shape: Tuple[int, int, int]  # (nx, ny, nz)
    orthogonal: bool = True
    bc: Tuple[int, int, int] = (0, 0, 0)  # 0 periodic, 1 Dirichlet
    fd_order: int = 12

    def __post_init__(self):
        self.latvec = np.asarray(self.latvec, dtype=np.float64).reshape(3, 3)
        self.shape = tuple(int(n) for n in self.shape)

    @property
    def lengths(self) -> np.ndarray:
        return np.linalg.norm(self.latvec, axis=1)

    @property
    def uvec(self) -> np.ndarray:
        return self.latvec / self.lengths[:, None]

    @property
    def intervals(self) -> np.ndarray:
        return np.array([n if b == 0 else n - 1 for n, b in zip(self.shape, self.bc)], dtype=np.float64)

    @property
    def spacing(self) -> np.ndarray:
        return self.lengths / self.intervals

    @property
    def nd(self) -> int:
        return int(np.prod(self.shape))

    @property
    def dV(self) -> float:
        return abs(float(np.linalg.det(self.latvec))) / float(np.prod(self.intervals))

    @property
    def lapc_T(self) -> np.ndarray:
        ui = np.linalg.inv(self.uvec)
        return ui.T @ ui

    def noncart_sphere_extent(self) -> np.ndarray:
        ui = np.linalg.inv(self.uvec)
        return np.sqrt((ui ** 2).sum(axis=0))

    def grid_points_cart(self) -> np.ndarray:
        """Cartesian coordinates of all grid points, x fastest (Nd x 3)."""
        nx, ny, nz = self.shape
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        nc = np.stack([i.ravel() * self.spacing[0], j.ravel() * self.spacing[1], k.ravel() * self.spacing[2]], 1)
        return nc @ self.uvec if not self.orthogonal else nc


def kpoints_mp(cell: Cell, kgrid: Sequence[int], shift=(0.0, 0.0, 0.0)):
    """Reduced Monkhorst-Pack k-points: (kcart [n,3], kred [n,3], weights [n]).

    kcart_d = kred_d * 2 pi / L_d (the reference's k units); -k is merged into k.
    """
    TOL = 1e-12
    L = cell.lengths
    two_pi = 2.0 * math.pi
    sums = two_pi / L
    kc, kr, w = [], [], []
    K = [int(v) for v in kgrid]
    starts = [-int(math.floor((n - 1) / 2.0)) for n in K]
    for n1 in range(starts[0], starts[0] + K[0]):
        for n2 in range(starts[1], starts[1] + K[1]):
            for n3 in range(starts[2], starts[2] + K[2]):
                red = []
                for n, Kd, s in ((n1, K[0], shift[0]), (n2, K[1], shift[1]), (n3, K[2], shift[2])):
                    v = n * 1.0 / Kd
                    v = math.fmod(v + s / Kd + 0.5 - TOL, 1.0) - 0.5 + TOL
                    red.append(v)
                cart = [red[d] * two_pi / L[d] for d in range(3)]
                found = -1
                for idx, kk in enumerate(kc):
                    ok = True
                    for d in range(3):
                        if not (abs(cart[d] + kk[d]) < TOL or abs(cart[d] + kk[d] - sums[d]) < TOL):
                            ok = False
                            break
                    if ok:
                        found = idx
                        break
                if found >= 0:
                    w[found] = 2.0
                else:
                    kc.append(cart)
                    kr.append(red)
                    w.append(1.0)
    return np.array(kc), np.array(kr), np.array(w)


_DIAMOND_FRAC = np.array([
    [0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5],
    [0.25, 0.25, 0.25], [0.75, 0.75, 0.25], [0.75, 0.25, 0.75], [0.25, 0.75, 0.75]])


def diamond_si(reps: int = 1, grid: int = 30, a: float = SI_A, displace: float = 0.0, strain=None,
               seed: int = 0, fd_order: int = 12) -> Tuple[Cell, np.ndarray]:
    """Conventional-cubic Si supercell (reps^3 cells, 8*reps^3 atoms) on a grid^3 mesh.

    displace: std-dev (Bohr) of seeded Gaussian displacements per coordinate.
    strain: None, a scalar (isotropic), or 3 diagonal strains (the cell stays orthogonal).
    """
    rng = np.random.default_rng(seed)
    frac = np.concatenate([(_DIAMOND_FRAC + np.array([i, j, k])) / reps
                           for i in range(reps) for j in range(reps) for k in range(reps)])
    eps = np.zeros(3) if strain is None else np.broadcast_to(np.asarray(strain, dtype=np.float64), (3,))
    L = a * reps * (1.0 + eps)
    latvec = np.diag(L)
    pos = frac * L
    if displace > 0:
        pos = pos + rng.normal(0.0, displace, size=pos.shape)
    pos = np.mod(pos, L)
    g = (grid, grid, grid) if np.isscalar(grid) else tuple(grid)
    return Cell(latvec, g, True, (0, 0, 0), fd_order), pos


def fcc_si_primitive(grid: int = 20, a: float = SI_A, fd_order: int = 12) -> Tuple[Cell, np.ndarray]:
    """Two-atom primitive FCC Si cell (non-orthogonal); positions in non-Cartesian coordinates."""
    latvec = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]])
    cell = Cell(latvec, (grid, grid, grid), False, (0, 0, 0), fd_order)
    frac = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
    return cell, frac * cell.lengths


def synthetic_veff(cell: Cell, positions: np.ndarray, depth: float = 1.2, width: float = 1.1,
                   noise: float = 0.0, seed: int = 0) -> np.ndarray:
    """Sum of Gaussian wells (-depth, std `width` Bohr) on every atom image, plus N(0, noise)."""
    pts = cell.grid_points_cart()
    L = cell.lengths
    pos_c = positions if cell.orthogonal else positions @ cell.uvec
    V = np.zeros(len(pts))
    reach = int(math.ceil(5.0 * width / L.min()))
    for p in pos_c:
        for i in range(-reach, reach + 1):
            for j in range(-reach, reach + 1):
                for k in range(-reach, reach + 1):
                    shift = np.array([i, j, k], dtype=np.float64) @ cell.latvec
                    d = pts - (p + shift)
                    V -= depth * np.exp(-(d * d).sum(1) / (2.0 * width * width))
    if noise > 0:
        V += np.random.default_rng(seed).normal(0.0, noise, size=V.shape)
    return V


def synthetic_veff_separable(cell: Cell, positions: np.ndarray, depth: float = 1.2, width: float = 1.1,
                             noise: float = 0.0, seed: int = 0) -> np.ndarray:
    """synthetic_veff for orthogonal cells, evaluated separably: every Gaussian well is a product of
    three periodic 1-D Gaussians (images -2..2 per axis), so large grids (90^3, 216 atoms) take
    seconds instead of minutes."""
    if not cell.orthogonal:
        raise ValueError("the separable form needs an orthogonal cell")
    nx, ny, nz = cell.shape
    h = cell.spacing
    L = cell.lengths
    axes = [np.arange(n) * h[d] for d, n in enumerate((nx, ny, nz))]
    V = np.zeros((nz, ny, nx))
    for p in positions:
        g = []
        for d in range(3):
            x = axes[d][:, None] - p[d] - L[d] * np.arange(-2, 3)[None, :]
            g.append(np.exp(-x * x / (2 * width * width)).sum(1))
        V -= depth * np.einsum("k,j,i->kji", g[2], g[1], g[0])
    V = V.ravel()
    if noise > 0:
        V += np.random.default_rng(seed).normal(0.0, noise, size=V.shape)
    return V


def random_orbitals(nd: int, nband: int, seed: int = 1, complex_: bool = False) -> np.ndarray:
    """Seeded U(-0.5, 0.5) orbitals, Fortran-ordered (nd, nband)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.5, 0.5, size=(nband, nd))
    if complex_:
        x = x + 1j * rng.uniform(-0.5, 0.5, size=(nband, nd))
    return np.asfortranarray(x.T)
