"""CPU restatement of the reference LYNX CheFSI hot path in numpy (FP64).

TEST INFRASTRUCTURE — the oracle.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may use it, and only as the checker.  The lynx_b200 product never
imports it.

Parity pinning: every function here is checked in tests/test_oracle_golden.py against
golden vectors produced by the reference's own code (tests/golden/make_golden.py runs
oracle/_ref/libref_lynx.so, i.e. the reference sources compiled unmodified).

Each function cites the reference file:line it restates (paths in the LYNX tree).
Orbitals are (Nd, ncol) arrays, grid index i + j*nx + k*nx*ny (x fastest).
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import scipy.linalg as sla
import scipy.optimize as sopt


# ---------------------------------------------------------------------------
# Finite-difference stencil (src/operators/FDStencil.cpp:7-180)
# ---------------------------------------------------------------------------

def fract(n: int, k: int) -> float:
    """n! / ((n-k)! (n+k)!)  (FDStencil.cpp:7-15)."""
    num = 1.0
    den = 1.0
    for i in range(n - k + 1, n + 1):
        num *= i
    for i in range(n + 1, n + k + 1):
        den *= i
    return num / den


def fd_weights(order: int) -> Tuple[np.ndarray, np.ndarray]:
    """First/second-derivative central weights w1, w2 (FDStencil.cpp:73-94)."""
    fdn = order // 2
    w1 = np.zeros(fdn + 1)
    w2 = np.zeros(fdn + 1)
    for p in range(1, fdn + 1):
        sgn = 1.0 if p % 2 == 1 else -1.0
        w1[p] = sgn * fract(fdn, p) / p
        w2[0] -= 2.0 / (p * p)
        w2[p] = sgn * 2.0 * fract(fdn, p) / (p * p)
    return w1, w2


def lattice_metrics(latvec: np.ndarray):
    """Unit lattice vectors, lapc_T = (U^-1)^T U^-1, jacobian (src/core/Lattice.cpp:13-51)."""
    L = np.linalg.norm(latvec, axis=1)
    U = latvec / L[:, None]
    Ui = np.linalg.inv(U)
    return U, Ui.T @ Ui, abs(np.linalg.det(latvec)), L


def stencil(latvec, shape, order, orthogonal=True, bc=(0, 0, 0)) -> Dict[str, np.ndarray]:
    """Grid-scaled coefficients and the max eigenvalue of -0.5 Lap
    (FDStencil.cpp:96-180; grid spacing FDGrid.cpp:18-37)."""
    latvec = np.asarray(latvec, dtype=np.float64)
    U, lapcT, jac, L = lattice_metrics(latvec)
    nint = np.array([n if b == 0 else n - 1 for n, b in zip(shape, bc)], dtype=np.float64)
    h = L / nint
    w1, w2 = fd_weights(order)
    fdn = order // 2
    out = {"dx": h, "dV": jac / nint.prod(), "w1": w1, "w2": w2}
    g = np.ones(3) if orthogonal else np.diag(lapcT)
    for d, ax in enumerate("xyz"):
        out["D1" + ax] = w1 / h[d]
        out["D2" + ax] = g[d] * w2 / h[d] ** 2
    if orthogonal:
        out["D2xy"] = np.zeros(fdn + 1)
        out["D2xz"] = np.zeros(fdn + 1)
        out["D2yz"] = np.zeros(fdn + 1)
        sc = [(n - n % 2) / n for n in shape]
        m = out["D2x"][0] + out["D2y"][0] + out["D2z"][0]
        for p in range(1, fdn + 1):
            m += 2.0 * sum(out["D2" + ax][p] * math.cos(math.pi * p * sc[d]) for d, ax in enumerate("xyz"))
        out["max_eigval"] = -0.5 * m
    else:
        out["D2xy"] = 2.0 * lapcT[0, 1] * w1 / h[0]
        out["D2xz"] = 2.0 * lapcT[0, 2] * w1 / h[0]
        out["D2yz"] = 2.0 * lapcT[1, 2] * w1 / h[1]
        m = abs(out["D2x"][0]) + abs(out["D2y"][0]) + abs(out["D2z"][0])
        for p in range(1, fdn + 1):
            m += 2.0 * (abs(out["D2x"][p]) + abs(out["D2y"][p]) + abs(out["D2z"][p]))
            m += 2.0 * (abs(out["D2xy"][p]) + abs(out["D2xz"][p]) + abs(out["D2yz"][p]))
        out["max_eigval"] = 0.5 * m
    return out


# ---------------------------------------------------------------------------
# Ghost-extended array (src/parallel/HaloExchange.cpp:34-189)
# ---------------------------------------------------------------------------

def extend(x3: np.ndarray, fdn: int, phases=None, bc=(0, 0, 0)) -> np.ndarray:
    """Ghost-padded copy of one column, array index [k, j, i].

    Periodic directions wrap (left ghost <- right interior, right ghost <- left interior),
    multiplied by e^{-ik_dL_d} (left) / e^{+ik_dL_d} (right) for Bloch phases; Dirichlet
    directions stay zero.  Wrapping runs z, then y, then x over the whole extended array,
    so corner ghosts carry the product of the phases (HaloExchange.cpp:46-95,136-189)."""
    nz, ny, nx = x3.shape
    xe = np.zeros((nz + 2 * fdn, ny + 2 * fdn, nx + 2 * fdn), dtype=x3.dtype)
    xe[fdn:fdn + nz, fdn:fdn + ny, fdn:fdn + nx] = x3
    ph = phases if phases is not None else [(1.0, 1.0)] * 3
    if bc[2] == 0:
        xe[:fdn] = xe[nz:nz + fdn] * ph[2][0]
        xe[nz + fdn:] = xe[fdn:2 * fdn] * ph[2][1]
    if bc[1] == 0:
        xe[:, :fdn] = xe[:, ny:ny + fdn] * ph[1][0]
        xe[:, ny + fdn:] = xe[:, fdn:2 * fdn] * ph[1][1]
    if bc[0] == 0:
        xe[:, :, :fdn] = xe[:, :, nx:nx + fdn] * ph[0][0]
        xe[:, :, nx + fdn:] = xe[:, :, fdn:2 * fdn] * ph[0][1]
    return xe


def bloch_phases(kpt, lengths):
    """(left, right) ghost multipliers per direction (HaloExchange.cpp:121-133)."""
    out = []
    for d in range(3):
        th = kpt[d] * lengths[d]
        out.append((complex(math.cos(th), -math.sin(th)), complex(math.cos(th), math.sin(th))))
    return out


# ---------------------------------------------------------------------------
# Hamiltonian (src/operators/Hamiltonian.cpp:64-267)
# ---------------------------------------------------------------------------

def h_local(psi, veff, shape, st, c=0.0, orthogonal=True, kpt=None, lengths=None, bc=(0, 0, 0)):
    """-0.5 Lap psi + (Veff + c) psi (Hamiltonian.cpp:127-174 orthogonal, 177-267 non-orthogonal)."""
    nx, ny, nz = shape
    fdn = len(st["D2x"]) - 1
    psi2 = psi.reshape(psi.shape[0], -1)
    out = np.zeros_like(psi2)
    ph = bloch_phases(kpt, lengths) if kpt is not None else None
    cx, cy, cz = st["D2x"], st["D2y"], st["D2z"]
    diag = cx[0] + cy[0] + cz[0]
    V = veff.reshape(nz, ny, nx)
    for n in range(psi2.shape[1]):
        x3 = psi2[:, n].reshape(nz, ny, nx)
        xe = extend(x3, fdn, ph, bc)
        s = (slice(fdn, fdn + nz), slice(fdn, fdn + ny), slice(fdn, fdn + nx))

        def sh(dk, dj, di):
            return xe[fdn + dk:fdn + dk + nz, fdn + dj:fdn + dj + ny, fdn + di:fdn + di + nx]

        lap = diag * xe[s]
        for p in range(1, fdn + 1):
            lap = lap + cx[p] * (sh(0, 0, p) + sh(0, 0, -p))
            lap = lap + cy[p] * (sh(0, p, 0) + sh(0, -p, 0))
            lap = lap + cz[p] * (sh(p, 0, 0) + sh(-p, 0, 0))
        if not orthogonal:
            for key, d1key, (a, b) in (("D2xy", "D1y", ((0, 0, 1), (0, 1, 0))),
                                        ("D2xz", "D1z", ((0, 0, 1), (1, 0, 0))),
                                        ("D2yz", "D1z", ((0, 1, 0), (1, 0, 0)))):
                c2 = st[key]
                d1 = st[d1key]
                if abs(c2[1]) <= 1e-30:
                    continue
                for p in range(1, fdn + 1):
                    for q in range(1, fdn + 1):
                        pa = tuple(p * v for v in a)
                        qb = tuple(q * v for v in b)
                        mixed = (sh(*[pa[i] + qb[i] for i in range(3)]) - sh(*[pa[i] - qb[i] for i in range(3)])
                                 - sh(*[-pa[i] + qb[i] for i in range(3)]) + sh(*[-pa[i] - qb[i] for i in range(3)]))
                        lap = lap + c2[p] * d1[q] * mixed
        out[:, n] = (-0.5 * lap + (V + c) * xe[s]).ravel()
    return out.reshape(psi.shape)


def nonlocal_apply(psi, hpsi, tab: dict, dV: float, kpt=None):
    """hpsi + Vnl psi with per-image Bloch factors (NonlocalProjector.cpp:121-347).

    tab: img_atom, img_ndc, img_shift, gpos, chi (per image ndc x nproj column-major),
    gamma (n_atom * nproj), nproj."""
    psi2 = psi.reshape(psi.shape[0], -1)
    out = np.array(hpsi, dtype=np.result_type(hpsi, psi)).reshape(psi2.shape)
    nproj = int(tab["nproj"])
    n_atom = len(tab["gamma"]) // nproj if nproj else 0
    ncol = psi2.shape[1]
    alpha = np.zeros((n_atom, nproj, ncol), dtype=out.dtype)
    offs = np.concatenate([[0], np.cumsum(tab["img_ndc"])])
    chis = []
    for i in range(len(tab["img_atom"])):
        ndc = int(tab["img_ndc"][i])
        chi = np.asarray(tab["chi"][offs[i] * nproj:(offs[i] + ndc) * nproj]).reshape(nproj, ndc).T
        chis.append(chi)
        g = tab["gpos"][offs[i]:offs[i] + ndc]
        fac = dV
        if kpt is not None:
            th = -float(np.dot(kpt, tab["img_shift"][i]))
            fac = complex(math.cos(th), math.sin(th)) * dV
        alpha[tab["img_atom"][i]] += fac * (chi.T @ psi2[g, :])
    alpha *= np.asarray(tab["gamma"]).reshape(n_atom, nproj)[:, :, None]
    for i in range(len(tab["img_atom"])):
        ndc = int(tab["img_ndc"][i])
        g = tab["gpos"][offs[i]:offs[i] + ndc]
        val = chis[i] @ alpha[tab["img_atom"][i]]
        if kpt is not None:
            th = -float(np.dot(kpt, tab["img_shift"][i]))
            val = complex(math.cos(th), -math.sin(th)) * val
        np.add.at(out, g, val)
    return out.reshape(np.shape(hpsi))


class Operator:
    """H = -0.5 Lap + Veff + Vnl for one cell (Hamiltonian::apply, Hamiltonian.cpp:22-28,64-75)."""

    def __init__(self, latvec, shape, order=12, orthogonal=True, tables: Optional[dict] = None, bc=(0, 0, 0)):
        self.latvec = np.asarray(latvec, dtype=np.float64)
        self.shape = tuple(shape)
        self.order = order
        self.orthogonal = orthogonal
        self.bc = bc
        self.st = stencil(self.latvec, shape, order, orthogonal, bc)
        self.dV = self.st["dV"]
        self.tab = tables
        self.lengths = np.linalg.norm(self.latvec, axis=1)
        self.nd = int(np.prod(shape))

    def apply(self, psi, veff, c=0.0, kpt=None):
        y = h_local(psi, veff, self.shape, self.st, c, self.orthogonal, kpt, self.lengths, self.bc)
        if self.tab is not None and len(self.tab["img_atom"]):
            y = nonlocal_apply(psi, y, self.tab, self.dV, kpt)
        return y


# ---------------------------------------------------------------------------
# CheFSI (src/solvers/EigenSolver.cpp:559-818)
# ---------------------------------------------------------------------------

def chebyshev_filter(H: Operator, X, veff, lc, emin, emax, degree, kpt=None):
    """Scaled three-term Chebyshev recurrence (EigenSolver.cpp:559-619)."""
    e = (emax - lc) / 2.0
    c = (emax + lc) / 2.0
    sigma1 = e / (emin - c)
    sigma = sigma1
    Y = (sigma / e) * (H.apply(X, veff, kpt=kpt) - c * X)
    Xold = np.array(X)
    for _ in range(2, degree + 1):
        sigma_new = 1.0 / (2.0 / sigma1 - sigma)
        gamma = 2.0 * sigma_new / e
        Xnew = gamma * (H.apply(Y, veff, kpt=kpt) - c * Y) - sigma * sigma_new * Xold
        Xold, Y = Y, Xnew
        sigma = sigma_new
    return Y


def orthogonalize(X, dV):
    """Cholesky-QR: S = dV X^H X = U^H U, X <- X U^-1 (EigenSolver.cpp:622-641)."""
    S = dV * (X.conj().T @ X)
    U = sla.cholesky(S, lower=False)
    return sla.solve_triangular(U, X.T, trans="T", lower=False).T if not np.iscomplexobj(X) else \
        sla.solve_triangular(U.T, X.T, lower=True).T


def project(H: Operator, X, veff, dV, kpt=None):
    """Hs = dV X^H H X, symmetrised (EigenSolver.cpp:644-660, symmetrize at :109-131)."""
    Hs = dV * (X.conj().T @ H.apply(X, veff, kpt=kpt))
    return 0.5 * (Hs + Hs.conj().T)


def solve(H: Operator, psi, veff, lc, emin, emax, degree=20, kpt=None):
    """One CheFSI pass (EigenSolver::solve_impl, EigenSolver.cpp:739-818).
    Returns (psi_out, eig, next lambda_cutoff)."""
    Y = chebyshev_filter(H, psi, veff, lc, emin, emax, degree, kpt)
    Y = orthogonalize(Y, H.dV)
    Hs = project(H, Y, veff, H.dV, kpt)
    eig, Q = np.linalg.eigh(Hs)
    return Y @ Q, eig, eig[-1] + 0.1


def _libc_rand_uniform(n: int, seed: int, complex_: bool):
    """Start vector with the C library's srand/rand (Lanczos.hpp:55-66, srand(1) at :112).

    For complex vectors the reference writes Complex(rand()/RAND_MAX, rand()/RAND_MAX);
    the order in which the two calls are evaluated is up to the compiler, and the GCC
    build of the reference evaluates the imaginary part's call first."""
    libc = ctypes.CDLL(None)
    libc.srand(ctypes.c_uint(seed))
    libc.rand.restype = ctypes.c_int
    RAND_MAX = 2147483647.0
    vals = np.array([libc.rand() / RAND_MAX for _ in range(2 * n if complex_ else n)])
    if complex_:
        return vals[1::2] + 1j * vals[0::2]
    return vals


def lanczos_bounds(H: Operator, veff, tol=1e-2, max_iter=1000, kpt=None):
    """Extreme eigenvalue estimates with the reference's margins (Lanczos.hpp:92-200)."""
    n = H.nd
    cplx = kpt is not None
    Vjm1 = _libc_rand_uniform(n, 1, cplx)
    Vjm1 = Vjm1 / np.linalg.norm(Vjm1)
    Vj = H.apply(Vjm1[:, None], veff, kpt=kpt)[:, 0]
    a = [float(np.real(np.vdot(Vjm1, Vj)))]
    Vj = Vj - a[0] * Vjm1
    b = [float(np.linalg.norm(Vj))]
    Vj = Vj / b[0]
    lo = hi = plo = phi = 0.0
    elo = ehi = tol + 1.0
    j = 0
    while (elo > tol or ehi > tol) and j < max_iter:
        Vp1 = H.apply(Vj[:, None], veff, kpt=kpt)[:, 0]
        a.append(float(np.real(np.vdot(Vj, Vp1))))
        Vp1 = Vp1 - (a[j + 1] * Vj + b[j] * Vjm1)
        Vjm1 = Vj
        b.append(float(np.linalg.norm(Vp1)))
        if b[j + 1] == 0.0:
            break
        Vj = Vp1 / b[j + 1]
        m = j + 2
        ev = sla.eigvalsh_tridiagonal(np.array(a[:m]), np.array(b[:m - 1]))
        lo, hi = ev[0], ev[-1]
        elo, ehi = abs(lo - plo), abs(hi - phi)
        plo, phi = lo, hi
        j += 1
    return lo - 0.1, hi * 1.01


# ---------------------------------------------------------------------------
# Occupations (src/electronic/Occupation.cpp:10-84)
# ---------------------------------------------------------------------------

def smearing(x, beta, fermi_dirac=True):
    """Fermi-Dirac with |x beta| > 50 clamped, or 0.5 erfc(beta x) (Occupation.cpp:10-35)."""
    x = np.asarray(x, dtype=np.float64)
    if fermi_dirac:
        t = x * beta
        with np.errstate(over="ignore"):
            f = 1.0 / (1.0 + np.exp(np.clip(t, -50.0, 50.0)))
        return np.where(t > 50.0, 0.0, np.where(t < -50.0, 1.0, f))
    from scipy.special import erfc
    return 0.5 * erfc(beta * x)


def fermi_level(eigs, weights, nelectron, beta, fermi_dirac=True):
    """Brent root of sum w f(eps - Ef) = N_e, brackets 10/beta then 100/beta (Occupation.cpp:48-84)."""
    eigs = np.asarray(eigs, dtype=np.float64)
    w = np.asarray(weights, dtype=np.float64)

    def res(ef):
        return float(np.sum(w * smearing(eigs - ef, beta, fermi_dirac)) - nelectron)

    a, b = eigs.min() - 10.0 / beta, eigs.max() + 10.0 / beta
    if res(a) * res(b) > 0:
        a, b = eigs.min() - 100.0 / beta, eigs.max() + 100.0 / beta
        if res(a) * res(b) > 0:
            raise ValueError("Cannot bracket Fermi level")
    return sopt.brentq(res, a, b, xtol=1e-14, rtol=4 * np.finfo(float).eps, maxiter=200)


# ---------------------------------------------------------------------------
# k-points (src/core/KPoints.cpp:8-80)
# ---------------------------------------------------------------------------

def kpoints(lengths, kgrid, shift=(0.0, 0.0, 0.0)):
    """Monkhorst-Pack points folded to [-0.5, 0.5), time-reversal pairs merged (weight 2)."""
    TOL = 1e-12
    lengths = np.asarray(lengths, dtype=np.float64)
    sums = 2 * np.pi / lengths
    kc, kr, w = [], [], []
    ranges = []
    for Kd in kgrid:
        s = -int(math.floor((Kd - 1) / 2.0))
        ranges.append(range(s, s + Kd))
    for n1 in ranges[0]:
        for n2 in ranges[1]:
            for n3 in ranges[2]:
                red = [math.fmod(n / Kd + sh / Kd + 0.5 - TOL, 1.0) - 0.5 + TOL
                       for n, Kd, sh in zip((n1, n2, n3), kgrid, shift)]
                cart = [red[d] * 2 * np.pi / lengths[d] for d in range(3)]
                hit = -1
                for i, q in enumerate(kc):
                    if all(abs(cart[d] + q[d]) < TOL or abs(cart[d] + q[d] - sums[d]) < TOL for d in range(3)):
                        hit = i
                        break
                if hit >= 0:
                    w[hit] = 2.0
                else:
                    kc.append(cart)
                    kr.append(red)
                    w.append(1.0)
    return np.array(kc), np.array(kr), np.array(w)


# ---------------------------------------------------------------------------
# Nonlocal force and energy (src/physics/Forces.cpp:509-797 compute_nonlocal_cpu,
# src/operators/Gradient.cpp:17-62; energy as documented at src/physics/GPUForce.cu:168-170)
# ---------------------------------------------------------------------------

def gradient(psi, shape, st, dim, kpt=None, lengths=None, bc=(0, 0, 0)):
    """D psi along lattice direction dim: sum_p D1[p] (x(+p) - x(-p)) on the ghost-extended
    block (Gradient.cpp:17-62; ghosts as HaloExchange::execute / execute_kpt)."""
    nx, ny, nz = shape
    c = st["D1" + "xyz"[dim]]
    fdn = len(c) - 1
    ph = bloch_phases(kpt, lengths) if kpt is not None else None
    psi2 = psi.reshape(psi.shape[0], -1)
    out = np.zeros_like(psi2)
    for n in range(psi2.shape[1]):
        xe = extend(psi2[:, n].reshape(nz, ny, nx), fdn, ph, bc)

        def sh(d):
            off = [0, 0, 0]
            off[2 - dim] = d  # arrays are (z, y, x)
            return xe[fdn + off[0]:fdn + off[0] + nz, fdn + off[1]:fdn + off[1] + ny, fdn + off[2]:fdn + off[2] + nx]

        g = np.zeros((nz, ny, nx), dtype=xe.dtype)
        for p in range(1, fdn + 1):
            g = g + c[p] * (sh(p) - sh(-p))
        out[:, n] = g.ravel()
    return out.reshape(psi.shape)


def projections(psi, tab: dict, dV: float, kpt=None):
    """alpha[atom, jp, n] = dV sum_img e^{-i k.R_img} chi_img^T psi (no Gamma), summed over the
    images of each atom in image order (Forces.cpp:701-722 real, :598-624 k-point)."""
    psi2 = psi.reshape(psi.shape[0], -1)
    nproj = int(tab["nproj"])
    n_atom = len(tab["gamma"]) // nproj if nproj else 0
    alpha = np.zeros((n_atom, nproj, psi2.shape[1]), dtype=np.result_type(psi2, 1.0))
    offs = np.concatenate([[0], np.cumsum(tab["img_ndc"])])
    for i in range(len(tab["img_atom"])):
        ndc = int(tab["img_ndc"][i])
        chi = np.asarray(tab["chi"][offs[i] * nproj:(offs[i] + ndc) * nproj]).reshape(nproj, ndc).T
        g = tab["gpos"][offs[i]:offs[i] + ndc]
        fac = dV
        if kpt is not None:
            th = -float(np.dot(kpt, tab["img_shift"][i]))
            fac = complex(math.cos(th), math.sin(th)) * dV
        alpha[tab["img_atom"][i]] += fac * (chi.T @ psi2[g, :])
    return alpha


def nonlocal_force(psi, occ, tab: dict, st, shape, dV, occfac=2.0, wk=1.0, kpt=None, lengths=None):
    """Nonlocal forces f[atom, dim] = -spn_fac wk sum_n g_n sum_jp Gamma Re(conj(alpha) beta_dim),
    spn_fac = 2 occfac, beta_dim = projections of D_dim psi (Forces.cpp:726-778, :662-684), and
    the nonlocal energy E = occfac wk sum_n g_n sum_jp Gamma |alpha|^2."""
    nproj = int(tab["nproj"])
    gam = np.asarray(tab["gamma"]).reshape(-1, nproj)[:, :, None]
    occ = np.asarray(occ, dtype=np.float64)[None, None, :]
    alpha = projections(psi, tab, dV, kpt)
    energy = occfac * wk * float(np.sum(occ * gam * np.abs(alpha) ** 2))
    f = np.zeros((alpha.shape[0], 3))
    for dim in range(3):
        beta = projections(gradient(psi, shape, st, dim, kpt, lengths), tab, dV, kpt)
        f[:, dim] = -2.0 * occfac * wk * np.sum(occ * gam * np.real(np.conj(alpha) * beta), axis=(1, 2))
    return f, energy


# ---------------------------------------------------------------------------
# Kinetic and nonlocal stress (src/physics/Stress.cpp:1041-1784 compute_nonlocal_kinetic_cpu:
# real path :1611-1729, k-point path :1229-1400, assembly :1732-1748), returned before the
# division by the cell measure, as Hamiltonian::compute_kinetic_nonlocal_stress_gpu returns it
# (src/operators/Hamiltonian.hpp:156-160; src/physics/GPUForce.cu:471-680).
# ---------------------------------------------------------------------------

VOIGT = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))


def cartesian_gradients(psi, cell, st, kpt=None):
    """Cartesian gradients [d/dx, d/dy, d/dz] of psi: lattice-direction FD gradients, mixed by
    uvec^-1 for non-orthogonal cells (Stress.cpp:1628-1640)."""
    G = [gradient(psi, cell.shape, st, d, kpt, cell.lengths, tuple(cell.bc)) for d in range(3)]
    if cell.orthogonal:
        return G
    ui = np.linalg.inv(cell.uvec)
    return [ui[a, 0] * G[0] + ui[a, 1] * G[1] + ui[a, 2] * G[2] for a in range(3)]


def weighted_projections(x, tab: dict, cell, dV: float, dim2: int, kpt=None):
    """beta[atom, jp, n] = dV sum_img e^{-i k.R_img} sum_g chi(g, jp) (r_g - R_img)_dim2 x(g), the
    relative position taken Cartesian (nonCart2Cart with uvec for non-orthogonal cells;
    Stress.cpp:1696-1717 real, :1350-1383 k-point)."""
    x2 = x.reshape(x.shape[0], -1)
    nproj = int(tab["nproj"])
    n_atom = len(tab["gamma"]) // nproj if nproj else 0
    beta = np.zeros((n_atom, nproj, x2.shape[1]), dtype=np.result_type(x2, 1.0))
    offs = np.concatenate([[0], np.cumsum(tab["img_ndc"])])
    nx, ny, _ = cell.shape
    h = cell.spacing
    uvec = cell.uvec
    for i in range(len(tab["img_atom"])):
        ndc = int(tab["img_ndc"][i])
        chi = np.asarray(tab["chi"][offs[i] * nproj:(offs[i] + ndc) * nproj]).reshape(nproj, ndc).T
        g = np.asarray(tab["gpos"][offs[i]:offs[i] + ndc])
        rel = np.stack([(g % nx) * h[0], ((g // nx) % ny) * h[1], (g // (nx * ny)) * h[2]], 1) - tab["img_coords"][i]
        if not cell.orthogonal:
            rel = rel @ uvec  # cart_j = sum_i nc_i uvec[i, j]
        w = rel[:, dim2]
        fac = dV
        if kpt is not None:
            th = -float(np.dot(kpt, tab["img_shift"][i]))
            fac = complex(math.cos(th), math.sin(th)) * dV
        beta[tab["img_atom"][i]] += fac * (chi.T @ (w[:, None] * x2[g, :]))
    return beta


def kinetic_nonlocal_stress(psi, occ, tab: dict, st, cell, dV, occfac=2.0, wk=1.0, kpt=None):
    """(stress_k[6], stress_nl[6]) in Voigt order xx, xy, xz, yy, yz, zz:
    stress_k = -occfac wk dV sum_n g_n Re <D_a psi_n, D_b psi_n>;
    stress_nl = -2 occfac wk sum_n g_n sum_jp Gamma Re(conj(alpha) beta_ab) - delta_ab E_nl,
    E_nl = occfac wk sum_n g_n sum_jp Gamma |alpha|^2."""
    occ = np.asarray(occ, dtype=np.float64)
    C = cartesian_gradients(psi, cell, st, kpt)
    sk = np.zeros(6)
    for v, (a, b) in enumerate(VOIGT):
        dots = np.real(np.sum(np.conj(C[a].reshape(C[a].shape[0], -1)) * C[b].reshape(C[b].shape[0], -1), axis=0))
        sk[v] = -occfac * wk * dV * float(np.sum(occ * dots))
    snl = np.zeros(6)
    energy = 0.0
    if tab is not None and len(tab["img_atom"]):
        nproj = int(tab["nproj"])
        gam = np.asarray(tab["gamma"]).reshape(-1, nproj)[:, :, None]
        oc = occ[None, None, :]
        alpha = projections(psi, tab, dV, kpt)
        energy = occfac * wk * float(np.sum(oc * gam * np.abs(alpha) ** 2))
        for v, (a, b) in enumerate(VOIGT):
            beta = weighted_projections(C[a], tab, cell, dV, b, kpt)
            snl[v] = -2.0 * occfac * wk * float(np.sum(oc * gam * np.real(np.conj(alpha) * beta)))
    snl[[0, 3, 5]] -= energy
    return sk, snl, energy
