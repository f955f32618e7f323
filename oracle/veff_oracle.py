"""CPU restatement of the reference's effective-potential build in numpy (FP64): GGA-PBE
exchange-correlation with the GGA divergence term, the AAR Poisson solver, and
V_eff = V_xc + phi (one spin channel).

TEST INFRASTRUCTURE — the oracle.  Only tests/ may use it, and only as the checker; the
lynx_b200 product never imports it.

Pinning: the Poisson solver is checked against the reference's own PoissonSolver compiled into
oracle/_ref (tests/test_oracle_veff.py); the functional against the known values in the
reference's XC unit tests (tests/unit/test_XCFunctional.cpp: Slater constants, PW92 correlation
at r_s = 2, PBE at zero gradient equal to LDA-PW).  The reference evaluates the functional with
libxc (XC_GGA_X_PBE + XC_GGA_C_PBE, src/xc/XCFunctional.cpp:42-54,230-245), which is not
available here, so the functional's parity with libxc itself is unpinned.
"""
from __future__ import annotations

import math

import numpy as np

from . import chefsi_oracle as O

# Published PBE / PW92 constants (Perdew, Burke, Ernzerhof 1996; Perdew, Wang 1992, zeta = 0).
KAPPA = 0.804
BETA = 0.06672455060314922
MU = BETA * math.pi ** 2 / 3.0
GAMMA = (1.0 - math.log(2.0)) / math.pi ** 2
PW_A, PW_A1 = 0.0310907, 0.21370
PW_B = (7.5957, 3.5876, 1.6382, 0.49294)


def lda_x(rho):
    """Uniform-gas exchange energy per particle, -(3/4)(3/pi)^(1/3) rho^(1/3)."""
    return -0.75 * (3.0 / math.pi) ** (1.0 / 3.0) * np.power(rho, 1.0 / 3.0)


def pw92_c(rs):
    """Uniform-gas correlation energy per particle of Perdew-Wang 1992, zeta = 0."""
    srs = np.sqrt(rs)
    den = 2.0 * PW_A * (PW_B[0] * srs + PW_B[1] * rs + PW_B[2] * rs * srs + PW_B[3] * rs * rs)
    return -2.0 * PW_A * (1.0 + PW_A1 * rs) * np.log(1.0 + 1.0 / den)


def pbe_energy_density(rho, sigma):
    """rho eps_xc(rho, sigma) of spin-unpolarised GGA-PBE; works on complex arguments (used for
    complex-step derivatives)."""
    r13 = np.power(rho, 1.0 / 3.0)
    kf = (3.0 * math.pi ** 2) ** (1.0 / 3.0) * r13
    s2 = sigma / (4.0 * kf * kf * rho * rho)
    fx = 1.0 + KAPPA - KAPPA / (1.0 + MU * s2 / KAPPA)
    ecu = pw92_c((3.0 / (4.0 * math.pi)) ** (1.0 / 3.0) / r13)
    t2 = sigma * math.pi / (16.0 * kf * rho * rho)
    A = (BETA / GAMMA) / (np.exp(-ecu / GAMMA) - 1.0)
    At2 = A * t2
    H = GAMMA * np.log(1.0 + (BETA / GAMMA) * t2 * (1.0 + At2) / (1.0 + At2 + At2 * At2))
    return rho * (lda_x(rho) * fx + ecu + H)


def pbe(rho, sigma):
    """exc (per particle), vrho = d(rho eps)/d rho, vsigma = d(rho eps)/d sigma; derivatives by the
    complex step (exact to rounding, independent of the GPU's dual numbers).  Points with
    rho <= 1e-14 give zeros."""
    rho = np.asarray(rho, dtype=np.float64)
    sigma = np.asarray(sigma, dtype=np.float64)
    ok = rho > 1e-14
    r = np.where(ok, rho, 1.0)
    s = np.where(ok, sigma, 0.0)
    h = 1e-30
    F = pbe_energy_density(r, s)
    vr = np.imag(pbe_energy_density(r + 1j * h * r, s)) / (h * r)
    vs = np.imag(pbe_energy_density(r.astype(complex), s + 1j * h)) / h
    exc = np.where(ok, F / r, 0.0)
    return exc, np.where(ok, vr, 0.0), np.where(ok, vs, 0.0)


def xc_gga_pbe(rho, H: "O.Operator", rho_core=None):
    """XCFunctional::evaluate_cpu, GGA branch (src/xc/XCFunctional.cpp:193-273) with this
    module's PBE: returns vxc, exc, dxcdgrho (= 2 vsigma)."""
    rho = np.asarray(rho, dtype=np.float64).ravel()
    if rho_core is not None:  # src/physics/EffectivePotential.cpp:127-134
        rho = np.maximum(rho + np.asarray(rho_core, dtype=np.float64).ravel(), 1e-14)
    st, shape, bc = H.st, H.shape, H.bc
    g = [O.gradient(rho[:, None], shape, st, d, bc=bc)[:, 0] for d in range(3)]
    if H.orthogonal:
        sigma = g[0] ** 2 + g[1] ** 2 + g[2] ** 2
    else:
        L = O.lattice_metrics(H.latvec)[1]
        sigma = (L[0, 0] * g[0] ** 2 + L[1, 1] * g[1] ** 2 + L[2, 2] * g[2] ** 2 + 2 * L[0, 1] * g[0] * g[1]
                 + 2 * L[0, 2] * g[0] * g[2] + 2 * L[1, 2] * g[1] * g[2])
    exc, vr, vs = pbe(rho, sigma)
    v2 = 2.0 * vs
    if H.orthogonal:
        f = [g[d] * v2 for d in range(3)]
    else:
        f = [(L[d, 0] * g[0] + L[d, 1] * g[1] + L[d, 2] * g[2]) * v2 for d in range(3)]
    vxc = vr.copy()
    for d in range(3):
        vxc -= O.gradient(f[d][:, None], shape, st, d, bc=bc)[:, 0]
    return vxc, exc, v2


def neg_laplacian(H: "O.Operator", x):
    """-Lap x (src/solvers/PoissonSolver.cpp:248-253)."""
    return 2.0 * O.h_local(np.asarray(x, dtype=np.float64).reshape(-1, 1), np.zeros(H.nd), H.shape, H.st, 0.0,
                           H.orthogonal, bc=H.bc)[:, 0]


def _gauss(A, b):
    """Partial-pivoting elimination skipping pivots below 1e-14 (src/core/NumericalMethods.cpp:84-120)."""
    A = A.copy()
    b = b.copy()
    n = len(b)
    for k in range(n):
        p = k + int(np.argmax(np.abs(A[k:, k])))  # first row of largest magnitude
        if p != k:
            A[[k, p]] = A[[p, k]]
            b[[k, p]] = b[[p, k]]
        d = A[k, k]
        if abs(d) < 1e-14:
            continue
        for i in range(k + 1, n):
            f = A[i, k] / d
            A[i, k + 1:] -= f * A[k, k + 1:]
            b[i] -= f * b[k]
    for k in range(n - 1, -1, -1):
        if abs(A[k, k]) < 1e-14:
            continue
        b[k] = (b[k] - A[k, k + 1:] @ b[k + 1:]) / A[k, k]
    return b


def poisson_aar(H: "O.Operator", b, phi0=None, tol=1e-8, max_iter=3000, m=7, p=6, omega=0.6, beta=0.6):
    """PoissonSolver::solve, CPU semantics (src/solvers/PoissonSolver.cpp:17-37 parameters,
    43-159 loop): returns (phi, iterations)."""
    b = np.asarray(b, dtype=np.float64).ravel()
    N = b.size
    phi = np.zeros(N) if phi0 is None else np.asarray(phi0, dtype=np.float64).ravel().copy()
    diag = H.st["D2x"][0] + H.st["D2y"][0] + H.st["D2z"][0]
    w = 1.0 if abs(diag) < 1e-14 else -1.0 / diag
    X = np.zeros((m, N))
    F = np.zeros((m, N))
    x_old = phi.copy()
    f_old = np.zeros(N)
    abs_tol = tol * math.sqrt(b @ b)
    r = b - neg_laplacian(H, phi)
    rn = abs_tol + 1.0
    it = 0
    while rn > abs_tol and it < max_iter:
        f = w * r
        if it > 0:
            c = (it - 1) % m
            X[c] = phi - x_old
            F[c] = f - f_old
        x_old = phi.copy()
        f_old = f.copy()
        if (it + 1) % p == 0 and it > 0:
            cols = min(it, m)
            Fc = F[:cols]
            gam = _gauss(Fc @ Fc.T, Fc @ f)
            phi = x_old + beta * f
            for j in range(cols):
                phi -= gam[j] * (X[j] + beta * F[j])
            r = b - neg_laplacian(H, phi)
            rn = math.sqrt(r @ r)
        else:
            phi = x_old + omega * f
            r = b - neg_laplacian(H, phi)
        it += 1
    return phi, it


def effective_potential(H: "O.Operator", rho, rho_b=None, rho_core=None, poisson_tol=1e-8, phi0=None):
    """EffectivePotential::compute, one spin channel (src/physics/EffectivePotential.cpp:44-71,
    73-177): returns veff, vxc, exc, phi, iterations."""
    rho = np.asarray(rho, dtype=np.float64).ravel()
    vxc, exc, _ = xc_gga_pbe(rho, H, rho_core)
    rhs = 4.0 * math.pi * rho
    if rho_b is not None:
        rhs = rhs + 4.0 * math.pi * np.asarray(rho_b, dtype=np.float64).ravel()
    rhs = rhs - rhs.sum() / rhs.size
    phi, it = poisson_aar(H, rhs, phi0, poisson_tol)
    phi = phi - phi.sum() / phi.size
    return vxc + phi, vxc, exc, phi, it
