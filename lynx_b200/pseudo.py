"""Pseudopotential input and nonlocal projector tables (set-up side, host, FP64).

Restates, in numpy, what the reference does before the hot path runs:

* ``read_psp8``          — Pseudopotential::load_psp8 (src/atoms/Pseudopotential.cpp:28-322):
                           radial grid, KB projectors p_l(r) = (r p_l)/r with the r=0
                           value copied from r=dr, KB energies Gamma[l][p], rc per l;
* ``spline_slopes`` / ``spline_eval`` — the cubic Hermite interpolation used for the
                           radial projectors (src/core/NumericalMethods.cpp:128-290):
                           slopes from the not-a-knot condition (de Boor, "A Practical
                           Guide to Splines", ch. IV), values clamped outside the grid;
* ``real_ylm``           — real spherical harmonics in the reference's sign and
                           normalisation conventions (src/core/math_utils.hpp:174-);
* ``nonlocal_tables``    — Crystal::compute_nloc_influence (src/atoms/Crystal.cpp:136-255)
                           and NonlocalProjector::setup (src/operators/NonlocalProjector.cpp:13-119):
                           every periodic image of every atom whose rc-sphere meets the
                           cell, its grid points, and chi[g, (l,p,m)] = Y_lm * p_l(|r|).

``synthetic_si_psp8`` writes a Si-like psp8 file (Z=14, Zval=4, lmax=2, 2 projectors per
channel, rc = 1.9/2.0/2.0 Bohr).  It stands in for the ONCV Si pseudopotential, which is
not available here; its radial shapes are smooth analytic functions chosen for this
project, not taken from any published pseudopotential.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence

import numpy as np

# ---------------------------------------------------------------------------
# psp8 files
# ---------------------------------------------------------------------------

_SYN_RC = (1.9, 2.0, 2.0)
_SYN_WIDTH = ((0.85, 0.5), (0.95, 0.55), (1.0, 0.6))
_SYN_EKB = ((4.2, 0.9), (1.6, -0.35), (-0.8, -0.05))


def _syn_projector(l: int, k: int, r: np.ndarray) -> np.ndarray:
    rc = _SYN_RC[l]
    s = _SYN_WIDTH[l][k]
    t = np.clip(r / rc, 0.0, 1.0)
    cut = (1.0 - t * t) ** 3
    poly = 1.0 if k == 0 else (1.0 - 1.6 * (r / rc) ** 2)
    p = (r ** l) * np.exp(-(r / s) ** 2) * poly * cut
    p[r >= rc] = 0.0
    return p


def synthetic_si_psp8(path: str, mmax: int = 600, dr: float = 0.01) -> str:
    """Write the Si-like synthetic psp8 file to `path` and return the path."""
    r = dr * np.arange(mmax)
    lines = ["Si-like synthetic psp8 (lynx_b200 test/benchmark input; not a physical pseudopotential)",
             "14.0000 4.0000 0", "8 11 2 4 %d 0.0" % mmax, "0.0 0.0 0.0", "2 2 2", "0"]
    for l in range(3):
        lines.append("%d %.12e %.12e" % (l, _SYN_EKB[l][0], _SYN_EKB[l][1]))
        u0 = r * _syn_projector(l, 0, r)
        u1 = r * _syn_projector(l, 1, r)
        for i in range(mmax):
            lines.append("%d %.12e %.15e %.15e" % (i + 1, r[i], u0[i], u1[i]))
    lines.append("4")
    zion, rloc = 4.0, 0.8
    for i in range(mmax):
        ri = r[i]
        v = -zion / ri * math.erf(ri / rloc) if ri > 0 else -zion * 2.0 / (math.sqrt(math.pi) * rloc)
        lines.append("%d %.12e %.15e" % (i + 1, ri, v))
    for i in range(mmax):
        lines.append("%d %.12e %.15e" % (i + 1, r[i], 4.0 * math.exp(-r[i] ** 2)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


@dataclasses.dataclass
class Psp8:
    zval: float
    lmax: int
    lloc: int
    ppl: List[int]
    r: np.ndarray
    udv: List[List[np.ndarray]]   # udv[l][p] = p_l(r)
    udv_d: List[List[np.ndarray]] # spline slopes
    gamma: List[List[float]]
    rc: List[float]

    @property
    def nproj_per_atom(self) -> int:
        return sum(self.ppl[l] * (2 * l + 1) for l in range(self.lmax + 1) if l != self.lloc)

    @property
    def rc_max(self) -> float:
        return max(self.rc) if self.rc else 0.0


def _fnum(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "E"))


def read_psp8(path: str) -> Psp8:
    """Parse the nonlocal part of a psp8 file the way the reference loader does."""
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)
    next(it)
    zval = _fnum(next(it).split()[1])
    h = next(it).split()
    pspcod, lmax, lloc, mmax = int(h[0]), int(h[2]), int(h[3]), int(h[4])
    if pspcod != 8:
        raise ValueError("only psp8 files are supported")
    next(it)
    ppl_tok = next(it).split()
    ppl = [int(ppl_tok[l]) for l in range(lmax + 1)]
    ext = int(next(it).split()[0])
    if ext >= 2:
        next(it)
    r = np.zeros(mmax)
    have_r = False
    udv: List[List[np.ndarray]] = [[] for _ in range(lmax + 1)]
    gamma: List[List[float]] = [[] for _ in range(lmax + 1)]
    for l in range(lmax + 1):
        hdr = next(it).split()
        nprj = ppl[l]
        if l != lloc and nprj > 0:
            gamma[l] = [_fnum(hdr[1 + p]) for p in range(nprj)]
            block = np.array([[_fnum(t) for t in next(it).split()[: 2 + nprj]] for _ in range(mmax)])
            ri = block[:, 1]
            if not have_r:
                r = ri.copy()
            vals = []
            for p in range(nprj):
                u = np.where(ri > 1e-10, block[:, 2 + p] / np.where(ri > 1e-10, ri, 1.0), 0.0)
                if mmax > 1:
                    u[0] = u[1]
                vals.append(u)
            udv[l] = vals
            have_r = True
        elif l == lloc:
            block = [next(it) for _ in range(mmax)]
            if not have_r:
                r = np.array([_fnum(b.split()[1]) for b in block])
            have_r = True
    if lloc > lmax:
        next(it)
        block = [next(it) for _ in range(mmax)]
        if not have_r:
            r = np.array([_fnum(b.split()[1]) for b in block])
    rc = []
    for l in range(lmax + 1):
        if ppl[l] > 0 and l != lloc:
            nz = np.nonzero(np.abs(udv[l][0]) > 1e-12)[0]
            rc.append(float(r[nz[-1]]) if len(nz) else float(r[-1]))
        else:
            rc.append(0.0)
    udv_d = [[spline_slopes(r, u) for u in udv[l]] for l in range(lmax + 1)]
    return Psp8(zval=zval, lmax=lmax, lloc=lloc, ppl=ppl, r=r, udv=udv, udv_d=udv_d, gamma=gamma, rc=rc)


# ---------------------------------------------------------------------------
# Cubic Hermite spline with not-a-knot slopes
# ---------------------------------------------------------------------------

def spline_slopes(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Node slopes s_i of the not-a-knot cubic spline through (x_i, y_i)."""
    n = len(x)
    s = np.zeros(n)
    if n < 2:
        return s
    if n == 2:
        s[:] = (y[1] - y[0]) / (x[1] - x[0])
        return s
    h = np.diff(x)
    dlt = np.diff(y) / h
    lo = np.zeros(n)   # sub-diagonal
    di = np.zeros(n)   # diagonal
    up = np.zeros(n)   # super-diagonal
    rhs = np.zeros(n)
    # first row: not-a-knot at x_1
    di[0] = h[1] * (h[0] + h[1])
    up[0] = (h[0] + h[1]) ** 2
    rhs[0] = dlt[0] * (3.0 * h[0] * h[1] + 2.0 * h[1] ** 2) + dlt[1] * h[0] ** 2
    # interior: continuity of the second derivative
    lo[1:-1] = h[1:]
    di[1:-1] = 2.0 * (h[:-1] + h[1:])
    up[1:-1] = h[:-1]
    rhs[1:-1] = 3.0 * (dlt[:-1] * h[1:] + dlt[1:] * h[:-1])
    # last row: not-a-knot at x_{n-2}
    h0, h1 = h[-2], h[-1]
    lo[-1] = (h0 + h1) ** 2
    di[-1] = h0 * (h0 + h1)
    rhs[-1] = dlt[-2] * h1 ** 2 + dlt[-1] * (3.0 * h0 * h1 + 2.0 * h0 ** 2)
    # Thomas algorithm
    cp = np.zeros(n)
    b = di[0]
    s[0] = rhs[0] / b
    for j in range(1, n):
        cp[j] = up[j - 1] / b
        b = di[j] - lo[j] * cp[j]
        if abs(b) < 1e-30:
            b = 1e-30
        s[j] = (rhs[j] - lo[j] * s[j - 1]) / b
    for j in range(n - 2, -1, -1):
        s[j] -= cp[j + 1] * s[j + 1]
    return s


def spline_eval(x: np.ndarray, y: np.ndarray, s: np.ndarray, xi: np.ndarray) -> np.ndarray:
    """Hermite cubic through (x, y) with slopes s, evaluated at xi (clamped outside [x0, x_end])."""
    xi = np.asarray(xi, dtype=np.float64)
    n = len(x)
    dx0 = x[1] - x[0]
    uniform = np.all(np.abs(np.diff(x) - dx0) <= 1e-10 * max(1.0, dx0))
    if uniform:
        j = np.floor((xi - x[0]) / dx0).astype(np.int64)
    else:
        j = np.searchsorted(x, xi, side="right") - 1
    j = np.clip(j, 0, n - 2)
    p1 = x[j]
    hinv = 1.0 / (x[j + 1] - p1)
    dy = (y[j + 1] - y[j]) * hinv
    a1 = s[j]
    a2 = hinv * (3.0 * dy - 2.0 * s[j] - s[j + 1])
    a3 = hinv * hinv * (-2.0 * dy + s[j] + s[j + 1])
    t = xi - p1
    out = ((a3 * t + a2) * t + a1) * t + y[j]
    out = np.where(xi <= x[0], y[0], out)
    out = np.where(xi >= x[-1], y[-1], out)
    return out


# ---------------------------------------------------------------------------
# Real spherical harmonics
# ---------------------------------------------------------------------------

def real_ylm(l: int, m: int, x, y, z, r) -> np.ndarray:
    """Real spherical harmonic Y_lm at Cartesian displacement (x, y, z), |.| = r."""
    x = np.asarray(x, dtype=np.float64)
    if l == 0:
        return np.full_like(x, 0.5 / math.sqrt(math.pi))
    rs = np.where(r < 1e-14, 1.0, r)
    xn, yn, zn = x / rs, y / rs, z / rs
    if l == 1:
        c = math.sqrt(3.0 / (4.0 * math.pi))
        v = {-1: c * yn, 0: c * zn, 1: c * xn}[m]
    elif l == 2:
        c1 = 0.5 * math.sqrt(15.0 / math.pi)
        c0 = 0.25 * math.sqrt(5.0 / math.pi)
        c2 = 0.25 * math.sqrt(15.0 / math.pi)
        v = {-2: c1 * xn * yn, -1: c1 * yn * zn, 0: c0 * (3.0 * zn * zn - 1.0), 1: c1 * xn * zn,
             2: c2 * (xn * xn - yn * yn)}[m]
    elif l == 3:
        x2, y2, z2 = xn * xn, yn * yn, zn * zn
        v = {-3: 0.25 * math.sqrt(35.0 / (2 * math.pi)) * yn * (3.0 * x2 - y2),
             -2: 0.5 * math.sqrt(105.0 / math.pi) * xn * yn * zn,
             -1: 0.25 * math.sqrt(21.0 / (2 * math.pi)) * yn * (5.0 * z2 - 1.0),
             0: 0.25 * math.sqrt(7.0 / math.pi) * zn * (5.0 * z2 - 3.0),
             1: 0.25 * math.sqrt(21.0 / (2 * math.pi)) * xn * (5.0 * z2 - 1.0),
             2: 0.25 * math.sqrt(105.0 / math.pi) * zn * (x2 - y2),
             3: 0.25 * math.sqrt(35.0 / (2 * math.pi)) * xn * (x2 - 3.0 * y2)}[m]
    else:
        raise NotImplementedError("l > 3")
    return np.where(r < 1e-14, 0.0, v)


# ---------------------------------------------------------------------------
# Nonlocal influence and projector tables
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class NonlocalTables:
    """Flattened projector tables in the layout of include/lynx_b200.h:lynx_set_nonlocal."""
    img_atom: np.ndarray    # int32 [n_img]
    img_ndc: np.ndarray     # int32 [n_img]
    img_shift: np.ndarray   # float64 [n_img, 3]
    img_coords: np.ndarray  # float64 [n_img, 3]
    gpos: np.ndarray        # int32 [sum ndc]
    chi: np.ndarray         # float64 [sum ndc*nproj] (per image, column-major ndc x nproj)
    atom_nproj: np.ndarray  # int32 [n_atom]
    gamma: np.ndarray       # float64 [sum nproj]

    @property
    def n_img(self) -> int:
        return len(self.img_atom)

    @property
    def n_atom(self) -> int:
        return len(self.atom_nproj)


def nonlocal_tables(cell, positions: np.ndarray, psp: Psp8) -> NonlocalTables:
    """Projector tables for atoms of one species at `positions` (n_atom x 3, Bohr).

    `cell` is a lynx_b200.cell.Cell.  Positions are Cartesian for orthogonal cells and
    non-Cartesian (fractional times |a_i|) for non-orthogonal cells, as in the reference.
    """
    positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    nx, ny, nz = cell.shape
    dx, dy, dz = cell.spacing
    L = cell.lengths
    rc = psp.rc_max
    ext = np.ones(3) if cell.orthogonal else cell.noncart_sphere_extent()
    nim = [int(math.ceil(rc * ext[d] / L[d])) if cell.bc[d] == 0 else 0 for d in range(3)]
    uvec = cell.uvec
    nproj = psp.nproj_per_atom
    img_atom, img_ndc, img_shift, img_coords, gpos_l, chi_l = [], [], [], [], [], []
    for ia, pos in enumerate(positions):
        for iz in range(-nim[2], nim[2] + 1):
            for iy in range(-nim[1], nim[1] + 1):
                for ix in range(-nim[0], nim[0] + 1):
                    img = pos + np.array([ix * L[0], iy * L[1], iz * L[2]])
                    if cell.orthogonal:
                        lo = np.ceil((img - rc) / cell.spacing).astype(int)
                        hi = np.floor((img + rc) / cell.spacing).astype(int)
                    else:
                        r_ext = rc * ext / cell.spacing
                        lo = np.ceil(img / cell.spacing - r_ext).astype(int)
                        hi = np.floor(img / cell.spacing + r_ext).astype(int)
                    lo = np.maximum(lo, 0)
                    hi = np.minimum(hi, np.array([nx - 1, ny - 1, nz - 1]))
                    if np.any(lo > hi):
                        continue
                    kk, jj, ii = np.meshgrid(np.arange(lo[2], hi[2] + 1), np.arange(lo[1], hi[1] + 1),
                                             np.arange(lo[0], hi[0] + 1), indexing="ij")
                    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
                    xr = ii * dx - img[0]
                    yr = jj * dy - img[1]
                    zr = kk * dz - img[2]
                    if cell.orthogonal:
                        cx, cy, cz = xr, yr, zr
                    else:
                        cx = xr * uvec[0, 0] + yr * uvec[1, 0] + zr * uvec[2, 0]
                        cy = xr * uvec[0, 1] + yr * uvec[1, 1] + zr * uvec[2, 1]
                        cz = xr * uvec[0, 2] + yr * uvec[1, 2] + zr * uvec[2, 2]
                    r2 = cx * cx + cy * cy + cz * cz
                    sel = r2 <= rc * rc
                    if not np.any(sel):
                        continue
                    ii, jj, kk = ii[sel], jj[sel], kk[sel]
                    cx, cy, cz = cx[sel], cy[sel], cz[sel]
                    rr = np.sqrt(cx * cx + cy * cy + cz * cz)
                    gp = ii + jj * nx + kk * nx * ny
                    cols = []
                    for l in range(psp.lmax + 1):
                        if l == psp.lloc:
                            continue
                        for p in range(psp.ppl[l]):
                            radial = spline_eval(psp.r, psp.udv[l][p], psp.udv_d[l][p], rr)
                            for m in range(-l, l + 1):
                                cols.append(real_ylm(l, m, cx, cy, cz, rr) * radial)
                    chi = np.stack(cols, axis=1) if cols else np.zeros((len(gp), 0))
                    img_atom.append(ia)
                    img_ndc.append(len(gp))
                    img_shift.append([ix * L[0], iy * L[1], iz * L[2]])
                    img_coords.append(img)
                    gpos_l.append(gp.astype(np.int32))
                    chi_l.append(np.asfortranarray(chi).ravel(order="F"))
    gam = []
    for _ in range(len(positions)):
        for l in range(psp.lmax + 1):
            if l == psp.lloc:
                continue
            for p in range(psp.ppl[l]):
                gam.extend([psp.gamma[l][p]] * (2 * l + 1))
    return NonlocalTables(
        img_atom=np.array(img_atom, dtype=np.int32),
        img_ndc=np.array(img_ndc, dtype=np.int32),
        img_shift=np.array(img_shift, dtype=np.float64).reshape(-1, 3),
        img_coords=np.array(img_coords, dtype=np.float64).reshape(-1, 3),
        gpos=np.concatenate(gpos_l) if gpos_l else np.zeros(0, np.int32),
        chi=np.concatenate(chi_l) if chi_l else np.zeros(0),
        atom_nproj=np.full(len(positions), nproj, dtype=np.int32),
        gamma=np.array(gam, dtype=np.float64),
    )
