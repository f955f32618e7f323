"""ctypes wrapper around oracle/_ref/libref_lynx.so — the reference LYNX CPU hot path.

TEST INFRASTRUCTURE.  The library is the reference's own EigenSolver / Hamiltonian /
NonlocalProjector / Occupation sources compiled by oracle/Makefile.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use it, as the
checker or the timed reference; the lynx_b200 package never imports it.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libref_lynx.so")

_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)
_d = ctypes.c_double
_i = ctypes.c_int

_SIG = {
    "ref_last_error": (ctypes.c_char_p, []),
    "ref_free": (None, []),
    "ref_setup": (_i, [_pd, _i, _i, _i, _i, _i, _i, _pd, ctypes.c_char_p]),
    "ref_setup_bc": (_i, [_pd, _i, _i, _i, _i, _i, _i, _pd, ctypes.c_char_p, _pi]),
    "ref_nd": (_i, []),
    "ref_dV": (_d, []),
    "ref_stencil": (_i, [_pd] * 12),
    "ref_lattice": (_i, [_pd, _pd, _pd, _pd]),
    "ref_nl_counts": (_i, [_pi, _pi, _pi, _pi]),
    "ref_nl_tables": (_i, [_pi, _pi, _pd, _pd, _pi, _pd, _pd, _pd]),
    "ref_h_apply": (_i, [_pd, _pd, _pd, _i, _d]),
    "ref_h_apply_kpt": (_i, [_pd, _pd, _pd, _i, _pd, _d]),
    "ref_nl_apply": (_i, [_pd, _pd, _i]),
    "ref_nl_apply_kpt": (_i, [_pd, _pd, _i, _pd]),
    "ref_chebyshev_filter": (_i, [_pd, _pd, _pd, _i, _d, _d, _d, _i]),
    "ref_chebyshev_filter_kpt": (_i, [_pd, _pd, _pd, _i, _d, _d, _d, _i, _pd]),
    "ref_solve": (_i, [_pd, _pd, _pd, _i, _d, _d, _d, _i]),
    "ref_solve_kpt": (_i, [_pd, _pd, _pd, _i, _d, _d, _d, _i, _pd]),
    "ref_lambda_cutoff": (_d, []),
    "ref_orthogonalize": (_i, [_pd, _i]),
    "ref_project": (_i, [_pd, _pd, _pd, _i]),
    "ref_diag": (_i, [_pd, _pd, _i]),
    "ref_rotate": (_i, [_pd, _pd, _i]),
    "ref_lanczos": (_i, [_pd, _pd, _pd, _d, _i]),
    "ref_lanczos_kpt": (_i, [_pd, _pd, _pd, _d, _i, _pd]),
    "ref_fermi_level": (_d, [_pd, _pd, _i, _d, _d, _i]),
    "ref_smearing": (_d, [_d, _d, _i]),
    "ref_kpoints": (_i, [_i, _i, _i, _pd, _pd, _pd, _pd, _i]),
    "ref_randomize": (None, [_pd, ctypes.c_long, ctypes.c_uint]),
    "ref_set_threads": (_i, [_i]),
    "ref_nonlocal_force": (_i, [_pd, _pd, _i, _i, _pd, _d, _pd]),
    "ref_kinetic_nonlocal_stress": (_i, [_pd, _pd, _i, _i, _pd, _d, _pd, _pd]),
    "ref_density": (_i, [_pd, _pd, _i, _i, _d, _pd]),
    "ref_poisson": (_i, [_pd, _pd, _d, _pi]),
    "ref_gradient": (_i, [_pd, _pd, _i]),
}

_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{REF_LIB} not built (make -C oracle)")
        l = ctypes.CDLL(REF_LIB)
        for k, (r, a) in _SIG.items():
            f = getattr(l, k)
            f.restype = r
            f.argtypes = a
        _lib = l
    return _lib


def _p(a):
    return a.ctypes.data_as(_pd)


def _ip(a):
    return a.ctypes.data_as(_pi)


def _chk(rc):
    if rc != 0:
        raise RuntimeError("reference oracle: " + lib().ref_last_error().decode())


class RefLynx:
    """One reference cell (grid, stencil, projectors) held by the oracle library."""

    def __init__(self, cell, positions: Optional[np.ndarray] = None, psp8_path: Optional[str] = None,
                 threads: Optional[int] = None):
        L = lib()
        if threads:
            L.ref_set_threads(int(threads))
        lat = np.ascontiguousarray(cell.latvec, dtype=np.float64)
        pos = np.ascontiguousarray(positions if positions is not None else np.zeros((0, 3)), dtype=np.float64)
        nx, ny, nz = cell.shape
        bc = np.ascontiguousarray(getattr(cell, "bc", (0, 0, 0)), dtype=np.int32)
        _chk(L.ref_setup_bc(_p(lat), 1 if cell.orthogonal else 0, nx, ny, nz, cell.fd_order, len(pos), _p(pos),
                            (psp8_path or "").encode(), _ip(bc)))
        self.nd = L.ref_nd()
        self.dV = L.ref_dV()
        self.cell = cell
        self.fdn = cell.fd_order // 2

    # -- set-up data ------------------------------------------------------
    def stencil(self) -> dict:
        n = self.fdn + 1
        keys = ("D2x", "D2y", "D2z", "D1x", "D1y", "D1z", "D2xy", "D2xz", "D2yz")
        out = {k: np.zeros(n) for k in keys}
        me = np.zeros(1)
        w1 = np.zeros(n)
        w2 = np.zeros(n)
        _chk(lib().ref_stencil(*[_p(out[k]) for k in keys], _p(me), _p(w1), _p(w2)))
        out["max_eigval"] = float(me[0])
        out["w1"] = w1
        out["w2"] = w2
        return out

    def nl_tables(self):
        ni, nt, npj, na = (ctypes.c_int() for _ in range(4))
        _chk(lib().ref_nl_counts(ctypes.byref(ni), ctypes.byref(nt), ctypes.byref(npj), ctypes.byref(na)))
        n_img, tot, nproj, n_atom = ni.value, nt.value, npj.value, na.value
        img_atom = np.zeros(n_img, np.int32)
        img_ndc = np.zeros(n_img, np.int32)
        img_shift = np.zeros((n_img, 3))
        img_coords = np.zeros((n_img, 3))
        gpos = np.zeros(tot, np.int32)
        chi = np.zeros(tot * nproj)
        gamma = np.zeros(n_atom * nproj)
        rc = np.zeros(1)
        _chk(lib().ref_nl_tables(_ip(img_atom), _ip(img_ndc), _p(img_shift), _p(img_coords), _ip(gpos), _p(chi),
                                 _p(gamma), _p(rc)))
        return dict(img_atom=img_atom, img_ndc=img_ndc, img_shift=img_shift, img_coords=img_coords, gpos=gpos,
                    chi=chi, gamma=gamma, nproj=nproj, n_atom=n_atom, rc=float(rc[0]))

    # -- operators -------------------------------------------------------------
    @staticmethod
    def _cols(psi, cplx=False):
        dt = np.complex128 if cplx else np.float64
        a = np.asarray(psi, dtype=dt)
        if a.ndim == 1:
            a = a[:, None]
        return np.asfortranarray(a)

    def h_apply(self, psi, veff, c=0.0):
        x = self._cols(psi)
        y = np.zeros_like(x, order="F")
        v = np.ascontiguousarray(veff, dtype=np.float64)
        _chk(lib().ref_h_apply(_p(x), _p(v), _p(y), x.shape[1], float(c)))
        return y

    def h_apply_kpt(self, psi, veff, kpt, c=0.0):
        x = self._cols(psi, True)
        y = np.zeros_like(x, order="F")
        v = np.ascontiguousarray(veff, dtype=np.float64)
        k = np.ascontiguousarray(kpt, dtype=np.float64)
        _chk(lib().ref_h_apply_kpt(x.ctypes.data_as(_pd), _p(v), y.ctypes.data_as(_pd), x.shape[1], _p(k), float(c)))
        return y

    def nl_apply(self, psi, hpsi):
        x = self._cols(psi)
        y = np.asfortranarray(np.array(hpsi, dtype=np.float64).reshape(x.shape, order="F"))
        _chk(lib().ref_nl_apply(_p(x), _p(y), x.shape[1]))
        return y

    def chebyshev_filter(self, X, veff, lc, emin, emax, degree):
        x = self._cols(X)
        y = np.zeros_like(x, order="F")
        v = np.ascontiguousarray(veff, dtype=np.float64)
        _chk(lib().ref_chebyshev_filter(_p(x), _p(y), _p(v), x.shape[1], lc, emin, emax, degree))
        return y

    def chebyshev_filter_kpt(self, X, veff, lc, emin, emax, degree, kpt):
        x = self._cols(X, True)
        y = np.zeros_like(x, order="F")
        v = np.ascontiguousarray(veff, dtype=np.float64)
        k = np.ascontiguousarray(kpt, dtype=np.float64)
        _chk(lib().ref_chebyshev_filter_kpt(x.ctypes.data_as(_pd), y.ctypes.data_as(_pd), _p(v), x.shape[1], lc,
                                            emin, emax, degree, _p(k)))
        return y

    def solve(self, psi, veff, lc, emin, emax, degree=20):
        x = self._cols(psi).copy(order="F")
        eig = np.zeros(x.shape[1])
        v = np.ascontiguousarray(veff, dtype=np.float64)
        _chk(lib().ref_solve(_p(x), _p(eig), _p(v), x.shape[1], lc, emin, emax, degree))
        return x, eig

    def solve_kpt(self, psi, veff, lc, emin, emax, degree, kpt):
        x = self._cols(psi, True).copy(order="F")
        eig = np.zeros(x.shape[1])
        v = np.ascontiguousarray(veff, dtype=np.float64)
        k = np.ascontiguousarray(kpt, dtype=np.float64)
        _chk(lib().ref_solve_kpt(x.ctypes.data_as(_pd), _p(eig), _p(v), x.shape[1], lc, emin, emax, degree, _p(k)))
        return x, eig

    def orthogonalize(self, X):
        x = self._cols(X).copy(order="F")
        _chk(lib().ref_orthogonalize(_p(x), x.shape[1]))
        return x

    def project(self, X, veff):
        x = self._cols(X)
        n = x.shape[1]
        hs = np.zeros((n, n), order="F")
        _chk(lib().ref_project(_p(x), _p(np.ascontiguousarray(veff, np.float64)), _p(hs), n))
        return hs

    def diag(self, Hs):
        h = np.asfortranarray(np.array(Hs, dtype=np.float64))
        eig = np.zeros(h.shape[0])
        _chk(lib().ref_diag(_p(h), _p(eig), h.shape[0]))
        return eig, h

    def rotate(self, X, Q):
        x = self._cols(X).copy(order="F")
        q = np.asfortranarray(np.array(Q, dtype=np.float64))
        _chk(lib().ref_rotate(_p(x), _p(q), x.shape[1]))
        return x

    def lanczos(self, veff, tol=1e-2, maxit=1000, kpt=None):
        lo = np.zeros(1)
        hi = np.zeros(1)
        v = np.ascontiguousarray(veff, dtype=np.float64)
        if kpt is None:
            _chk(lib().ref_lanczos(_p(v), _p(lo), _p(hi), tol, maxit))
        else:
            k = np.ascontiguousarray(kpt, dtype=np.float64)
            _chk(lib().ref_lanczos_kpt(_p(v), _p(lo), _p(hi), tol, maxit, _p(k)))
        return float(lo[0]), float(hi[0])

    # -- consumers of the orbitals (Nspin = 1: occfac = 2; one k-point of weight wk) ----------
    def _orb_args(self, psi, occ, kpt):
        cplx = kpt is not None
        x = self._cols(psi, cplx)
        o = np.ascontiguousarray(occ, dtype=np.float64)
        if o.shape[0] != x.shape[1]:
            raise ValueError("one occupation per orbital column is needed")
        k = np.ascontiguousarray(kpt if cplx else np.zeros(3), dtype=np.float64)
        return x, o, k, cplx

    def nonlocal_force(self, psi, occ, kpt=None, wk=1.0):
        """Forces::compute_nonlocal_cpu (src/physics/Forces.cpp:509-797): n_atom x 3."""
        x, o, k, cplx = self._orb_args(psi, occ, kpt)
        n_atom = ctypes.c_int()
        ni, nt, npj = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _chk(lib().ref_nl_counts(ctypes.byref(ni), ctypes.byref(nt), ctypes.byref(npj), ctypes.byref(n_atom)))
        f = np.zeros(3 * n_atom.value)
        _chk(lib().ref_nonlocal_force(x.ctypes.data_as(_pd), _p(o), x.shape[1], int(cplx), _p(k), float(wk), _p(f)))
        return f.reshape(-1, 3)

    def kinetic_nonlocal_stress(self, psi, occ, kpt=None, wk=1.0):
        """Stress::compute_nonlocal_kinetic_cpu (src/physics/Stress.cpp:1041-1784), before the
        division by the cell measure: (stress_k, stress_nl), Voigt xx, xy, xz, yy, yz, zz."""
        x, o, k, cplx = self._orb_args(psi, occ, kpt)
        sk = np.zeros(6)
        snl = np.zeros(6)
        _chk(lib().ref_kinetic_nonlocal_stress(x.ctypes.data_as(_pd), _p(o), x.shape[1], int(cplx), _p(k), float(wk),
                                               _p(sk), _p(snl)))
        return sk, snl

    def density(self, psi, occ, complex_=False, wk=1.0):
        """ElectronDensity::compute (src/electronic/ElectronDensity.cpp:55-172), Nspin = 1:
        rho = sum_n 2 wk occ[n] |psi_n|^2."""
        x = self._cols(psi, complex_)
        o = np.ascontiguousarray(occ, dtype=np.float64)
        rho = np.zeros(self.nd)
        _chk(lib().ref_density(x.ctypes.data_as(_pd), _p(o), x.shape[1], int(complex_), float(wk), _p(rho)))
        return rho

    def poisson(self, rhs, phi0=None, tol=1e-8):
        """PoissonSolver::solve (src/solvers/PoissonSolver.cpp:43-159): -Lap phi = rhs from phi0
        (zeros); returns (phi, iterations)."""
        b = np.ascontiguousarray(rhs, dtype=np.float64).ravel()
        phi = np.zeros(self.nd) if phi0 is None else np.ascontiguousarray(phi0, dtype=np.float64).ravel().copy()
        it = ctypes.c_int(0)
        _chk(lib().ref_poisson(_p(b), _p(phi), float(tol), ctypes.byref(it)))
        return phi, it.value

    def gradient(self, x, dim):
        """Gradient::apply of one field along direction dim (src/operators/Gradient.cpp:17-62)."""
        v = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.zeros(self.nd)
        _chk(lib().ref_gradient(_p(v), _p(y), int(dim)))
        return y

    def kpoints(self, kgrid, shift=(0.0, 0.0, 0.0)):
        n = int(np.prod(kgrid))
        kc = np.zeros((n, 3))
        kr = np.zeros((n, 3))
        w = np.zeros(n)
        s = np.ascontiguousarray(shift, dtype=np.float64)
        m = lib().ref_kpoints(int(kgrid[0]), int(kgrid[1]), int(kgrid[2]), _p(s), _p(kc), _p(kr), _p(w), n)
        return kc[:m], kr[:m], w[:m]


def fermi_level(eigs, weights, nelectron, beta, fermi_dirac=True):
    e = np.ascontiguousarray(eigs, dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    return float(lib().ref_fermi_level(_p(e), _p(w), len(e), float(nelectron), float(beta), 1 if fermi_dirac else 0))


def smearing(x, beta, fermi_dirac=True):
    return float(lib().ref_smearing(float(x), float(beta), 1 if fermi_dirac else 0))


def set_threads(n: int) -> int:
    return int(lib().ref_set_threads(int(n)))
