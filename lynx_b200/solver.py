"""Python mirror of the reference operator API on top of the lynx_b200 C ABI.

Mirrors the pybind11 layer of the reference (python/src/bind_solvers.cpp:54-114,
python/src/bind_operators.cpp:51-71) and python/lynx/ops/hamiltonian.py:
same method names, argument meaning and return values.

Orbitals can be passed two ways:
  * host numpy arrays of shape (Nd, nband) (Fortran order, like the reference binding),
    copied to the device for the call and back;
  * device-resident torch tensors of shape (nband, Nd) (contiguous, i.e. column-major
    Nd x nband), float64 or complex128, used in place on torch's current CUDA stream.
torch is used for device memory and streams only; every operator runs in liblynxb200.so.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr
from .cell import Cell
from .pseudo import NonlocalTables

_PREC = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}
_SMEAR = {"fermi-dirac": _lib.SMEAR_FERMI_DIRAC, "fd": _lib.SMEAR_FERMI_DIRAC,
          "gaussian": _lib.SMEAR_GAUSSIAN}


def _torch():
    import torch
    return torch


def _is_torch(x) -> bool:
    try:
        import torch
        return isinstance(x, torch.Tensor)
    except ImportError:  # pragma: no cover
        return False


def _dev_ptr(t) -> int:
    if not t.is_cuda:
        raise ValueError("device tensors must live on a CUDA device")
    if not t.is_contiguous():
        raise ValueError("device tensors must be contiguous")
    return t.data_ptr()


class Context:
    """One cell (grid, lattice, FD stencil, boundary conditions, projectors) on one GPU.

    Replaces the reference's FDGrid/Lattice/FDStencil/HaloExchange set-up and
    Hamiltonian::setup_gpu (see include/lynx_b200.h:lynx_create)."""

    def __init__(self, cell: Cell, device: int = 0):
        self.lib = _lib.load()
        self.cell = cell
        self.device = device
        h = ctypes.c_void_p()
        lat = np.ascontiguousarray(cell.latvec, dtype=np.float64)
        bc = np.ascontiguousarray(cell.bc, dtype=np.int32)
        nx, ny, nz = cell.shape
        check(self.lib.lynx_create(ctypes.byref(h), device, nx, ny, nz, cell.fd_order, dptr(lat),
                                   1 if cell.orthogonal else 0, iptr(bc)))
        self._h = h
        nd = ctypes.c_int()
        dv = ctypes.c_double()
        me = ctypes.c_double()
        check(self.lib.lynx_grid_info(self._h, ctypes.byref(nd), ctypes.byref(dv), ctypes.byref(me)))
        self.nd = nd.value
        self.dV = dv.value
        self.max_eigval_half_lap = me.value
        self.has_nonlocal = False
        self.kpt = np.zeros(3)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.lynx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync_stream(self):
        """Point the context at torch's current CUDA stream."""
        torch = _torch()
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.lib.lynx_set_stream(self._h, ctypes.c_void_p(s)))

    def set_stream(self, stream):
        """Put the context's work on `stream` (a torch.cuda.Stream or a raw cudaStream_t)."""
        raw = getattr(stream, "cuda_stream", stream)
        check(self.lib.lynx_set_stream(self._h, ctypes.c_void_p(int(raw))))

    def set_option(self, option: int, value: int):
        check(self.lib.lynx_set_option(self._h, int(option), int(value)))

    def stencil_coeffs(self) -> dict:
        n = self.cell.fd_order // 2 + 1
        out = {k: np.zeros(n) for k in ("D2x", "D2y", "D2z", "D2xy", "D2xz", "D2yz", "D1x", "D1y", "D1z")}
        check(self.lib.lynx_stencil_coeffs(self._h, *[dptr(out[k]) for k in
                                                      ("D2x", "D2y", "D2z", "D2xy", "D2xz", "D2yz", "D1x", "D1y", "D1z")]))
        return out

    def set_nonlocal(self, tab: Optional[NonlocalTables]):
        if tab is None or tab.n_img == 0:
            check(self.lib.lynx_set_nonlocal(self._h, 0, None, None, None, None, None, 0, None, None))
            self.has_nonlocal = False
            return
        a = np.ascontiguousarray(tab.img_atom, np.int32)
        n = np.ascontiguousarray(tab.img_ndc, np.int32)
        s = np.ascontiguousarray(tab.img_shift, np.float64)
        g = np.ascontiguousarray(tab.gpos, np.int32)
        c = np.ascontiguousarray(tab.chi, np.float64)
        npj = np.ascontiguousarray(tab.atom_nproj, np.int32)
        gm = np.ascontiguousarray(tab.gamma, np.float64)
        check(self.lib.lynx_set_nonlocal(self._h, tab.n_img, iptr(a), iptr(n), dptr(s), iptr(g), dptr(c),
                                         tab.n_atom, iptr(npj), dptr(gm)))
        self.has_nonlocal = True
        self.n_atom = int(tab.n_atom)
        self.img_coords = np.ascontiguousarray(tab.img_coords, dtype=np.float64).reshape(-1, 3)

    def set_kpoint(self, kcart):
        k = np.ascontiguousarray(kcart, dtype=np.float64).reshape(3)
        check(self.lib.lynx_set_kpoint(self._h, dptr(k)))
        self.kpt = k.copy()


class _DeviceArgs:
    """Moves host numpy orbitals to the device for one call and back."""

    def __init__(self, ctx: Context, psi, complex_: bool):
        torch = _torch()
        self.host = not _is_torch(psi)
        self.complex = complex_
        if self.host:
            arr = np.asarray(psi)
            self.one_d = arr.ndim == 1
            arr2 = arr.reshape(arr.shape[0], -1, order="F")
            if arr2.shape[0] != ctx.nd:
                raise ValueError(f"psi has {arr2.shape[0]} rows, the grid has {ctx.nd} points")
            dt = np.complex128 if complex_ else np.float64
            cols = np.ascontiguousarray(arr2.T.astype(dt, copy=False))
            self.t = torch.from_numpy(cols).to(f"cuda:{ctx.device}")
        else:
            self.one_d = psi.dim() == 1
            self.t = psi.reshape(1, -1) if self.one_d else psi
            if self.t.shape[-1] != ctx.nd:
                raise ValueError(f"psi rows {self.t.shape[-1]} != grid points {ctx.nd}")
        self.ncol = self.t.shape[0]

    def like(self):
        return _torch().empty_like(self.t)

    def out(self, t):
        if self.host:
            a = t.cpu().numpy().T
            a = np.asfortranarray(a)
            return a[:, 0] if self.one_d else a
        return t.reshape(-1) if self.one_d else t


def _veff_dev(ctx: Context, Veff):
    torch = _torch()
    if _is_torch(Veff):
        v = Veff.to(device=f"cuda:{ctx.device}", dtype=torch.float64).contiguous()
    else:
        v = torch.from_numpy(np.ascontiguousarray(Veff, dtype=np.float64)).to(f"cuda:{ctx.device}")
    if v.numel() != ctx.nd:
        raise ValueError("Veff must have Nd entries")
    return v


class NonlocalProjector:
    """Vnl apply (NonlocalProjector::apply / apply_kpt): returns hpsi + Vnl psi."""

    def __init__(self, ctx: Context, tables: Optional[NonlocalTables] = None):
        self.ctx = ctx
        if tables is not None:
            ctx.set_nonlocal(tables)

    def total_nproj(self) -> int:
        return 0

    def apply(self, psi, hpsi, kpt: bool = False):
        ctx = self.ctx
        ctx.sync_stream()
        a = _DeviceArgs(ctx, psi, kpt)
        h = _DeviceArgs(ctx, hpsi, kpt)
        fn = ctx.lib.lynx_nonlocal_apply_kpt if kpt else ctx.lib.lynx_nonlocal_apply
        check(fn(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), ctypes.c_void_p(_dev_ptr(h.t)), a.ncol, ctx.nd))
        return h.out(h.t)

    def force(self, psi, occ, occfac: float = 2.0, kpt: bool = False, wk: float = 1.0):
        """Nonlocal forces (n_atom x 3, Ha/Bohr along the lattice directions) and energy of the
        orbitals psi with occupations occ (Hamiltonian::compute_nonlocal_force_gpu /
        _kpt_gpu; the formula of Forces.cpp:509-797).  k-point: spn_fac * wk = 2 occfac wk."""
        ctx = self.ctx
        ctx.sync_stream()
        a = _DeviceArgs(ctx, psi, kpt)
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        if occ.shape[0] != a.ncol:
            raise ValueError("one occupation per orbital column is needed")
        na = getattr(ctx, "n_atom", 0)
        f = np.zeros(3 * max(na, 1))
        e = np.zeros(1)
        if kpt:
            check(ctx.lib.lynx_nonlocal_force_kpt(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), a.ncol, ctx.nd,
                                                  dptr(occ), 2.0 * occfac * wk, dptr(f), dptr(e)))
        else:
            check(ctx.lib.lynx_nonlocal_force(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), a.ncol, ctx.nd, dptr(occ),
                                              occfac * wk, dptr(f), dptr(e)))
        return f[:3 * na].reshape(na, 3), float(e[0])

    def stress(self, psi, occ, occfac: float = 2.0, kpt: bool = False, wk: float = 1.0):
        """Kinetic and nonlocal stress (Voigt xx, xy, xz, yy, yz, zz) of the orbitals psi with
        occupations occ, before the division by the cell measure
        (Hamiltonian::compute_kinetic_nonlocal_stress_gpu / _kpt_gpu; the formula of
        Stress.cpp:1041-1784).  Returns (stress_k, stress_nl)."""
        ctx = self.ctx
        ctx.sync_stream()
        a = _DeviceArgs(ctx, psi, kpt)
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        if occ.shape[0] != a.ncol:
            raise ValueError("one occupation per orbital column is needed")
        sk = np.zeros(6)
        snl = np.zeros(6)
        pos = getattr(ctx, "img_coords", None) if ctx.has_nonlocal else None
        pp = dptr(pos) if pos is not None else None
        if kpt:
            check(ctx.lib.lynx_kinetic_nonlocal_stress_kpt(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), a.ncol, ctx.nd,
                                                           dptr(occ), 2.0 * occfac * wk, pp, dptr(sk), dptr(snl)))
        else:
            check(ctx.lib.lynx_kinetic_nonlocal_stress(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), a.ncol, ctx.nd,
                                                       dptr(occ), occfac * wk, pp, dptr(sk), dptr(snl)))
        return sk, snl


class Hamiltonian:
    """H psi = -0.5 Lap psi + Veff psi + Vnl psi (+ shift psi).

    Mirrors lynx.ops.Hamiltonian (python/lynx/ops/hamiltonian.py:1-64) and the C++
    Hamiltonian::apply / apply_kpt."""

    def __init__(self, ctx: Context, Veff=None):
        self.ctx = ctx
        self._Veff = None if Veff is None else np.asarray(Veff, dtype=np.float64)

    def set_potential(self, Veff):
        self._Veff = Veff

    def apply(self, psi, Veff=None, shift: float = 0.0):
        return self._apply(psi, Veff, shift, False)

    def apply_kpt(self, psi, Veff=None, shift: float = 0.0):
        return self._apply(psi, Veff, shift, True)

    def __call__(self, psi, Veff=None, shift: float = 0.0):
        return self.apply(psi, Veff, shift)

    def __matmul__(self, psi):
        return self.apply(psi)

    def _apply(self, psi, Veff, shift, kpt):
        ctx = self.ctx
        V = self._Veff if Veff is None else Veff
        if V is None:
            raise ValueError("No effective potential set. Call set_potential() first.")
        ctx.sync_stream()
        a = _DeviceArgs(ctx, psi, kpt)
        v = _veff_dev(ctx, V)
        y = a.like()
        fn = ctx.lib.lynx_hamiltonian_apply_kpt if kpt else ctx.lib.lynx_hamiltonian_apply
        check(fn(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), ctypes.c_void_p(v.data_ptr()),
                 ctypes.c_void_p(_dev_ptr(y)), a.ncol, ctx.nd, float(shift)))
        return a.out(y)


class EigenSolver:
    """Chebyshev-filtered subspace iteration (EigenSolver::solve / solve_kpt / lanczos_bounds).

    solve(psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree=20) -> (psi_out, eig),
    the signature of the reference binding (python/src/bind_solvers.cpp:54-114).  Host numpy
    psi is copied (the reference binding copies too); a device torch tensor is updated in place
    and returned."""

    def __init__(self, ctx: Context, precision: str = "fp64"):
        self.ctx = ctx
        self.precision = precision
        self._lambda_cutoff = 0.0

    def lambda_cutoff(self) -> float:
        return self._lambda_cutoff

    def set_lambda_cutoff(self, lc: float):
        self._lambda_cutoff = float(lc)

    def _solve(self, psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree, precision, kpt):
        ctx = self.ctx
        prec = _PREC[precision or self.precision]
        ctx.sync_stream()
        a = _DeviceArgs(ctx, psi, kpt)
        v = _veff_dev(ctx, Veff)
        eig = np.zeros(a.ncol)
        lc_out = ctypes.c_double()
        fn = ctx.lib.lynx_eigensolver_solve_kpt if kpt else ctx.lib.lynx_eigensolver_solve
        check(fn(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), dptr(eig), ctypes.c_void_p(v.data_ptr()), a.ncol,
                 ctx.nd, float(lambda_cutoff), float(eigval_min), float(eigval_max), int(cheb_degree), prec,
                 ctypes.byref(lc_out)))
        self._lambda_cutoff = lc_out.value
        return a.out(a.t), eig

    def solve(self, psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree: int = 20,
              precision: Optional[str] = None):
        return self._solve(psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree, precision, False)

    def solve_kpt(self, psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree: int = 20,
                  precision: Optional[str] = None):
        return self._solve(psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree, precision, True)

    def solve_density(self, psi, Veff, lambda_cutoff, eigval_min, eigval_max, cheb_degree: int = 20,
                      nelectron: float = 0.0, beta: float = 1000.0, smearing: str = "fermi-dirac",
                      weight: float = 2.0, rho=None, precision: Optional[str] = None):
        """One CheFSI pass, then the Fermi level, occupations and electron density of the new
        orbitals (lynx_eigensolver_solve_density; real orbitals, one spin channel and k-point).
        rho: a device tensor of Nd doubles to write, or None for a new one.  Returns
        (psi_out, eig, rho, ef)."""
        ctx = self.ctx
        torch = _torch()
        prec = _PREC[precision or self.precision]
        ctx.sync_stream()
        a = _DeviceArgs(ctx, psi, False)
        v = _veff_dev(ctx, Veff)
        if rho is None:
            rho = torch.empty(ctx.nd, dtype=torch.float64, device=f"cuda:{ctx.device}")
        eig = np.zeros(a.ncol)
        lc_out, ef = ctypes.c_double(), ctypes.c_double()
        sm = _SMEAR[smearing]
        check(ctx.lib.lynx_eigensolver_solve_density(
            ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), dptr(eig), ctypes.c_void_p(v.data_ptr()), a.ncol, ctx.nd,
            float(lambda_cutoff), float(eigval_min), float(eigval_max), int(cheb_degree), prec, ctypes.byref(lc_out),
            float(nelectron), float(beta), sm, float(weight), ctypes.c_void_p(_dev_ptr(rho)), ctypes.byref(ef)))
        self._lambda_cutoff = lc_out.value
        return a.out(a.t), eig, rho, ef.value

    def chebyshev_filter(self, X, Veff, lambda_cutoff, eigval_min, eigval_max, degree: int = 20,
                         precision: Optional[str] = None, kpt: bool = False):
        ctx = self.ctx
        ctx.sync_stream()
        a = _DeviceArgs(ctx, X, kpt)
        v = _veff_dev(ctx, Veff)
        y = a.like()
        fn = ctx.lib.lynx_chebyshev_filter_kpt if kpt else ctx.lib.lynx_chebyshev_filter
        check(fn(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), ctypes.c_void_p(_dev_ptr(y)),
                 ctypes.c_void_p(v.data_ptr()), a.ncol, ctx.nd, float(lambda_cutoff), float(eigval_min),
                 float(eigval_max), int(degree), _PREC[precision or self.precision]))
        return a.out(y)

    def lanczos_bounds(self, Veff, tol: float = 1e-2, max_iter: int = 1000, kpt: bool = False) -> Tuple[float, float]:
        ctx = self.ctx
        ctx.sync_stream()
        v = _veff_dev(ctx, Veff)
        lo, hi = ctypes.c_double(), ctypes.c_double()
        fn = ctx.lib.lynx_lanczos_bounds_kpt if kpt else ctx.lib.lynx_lanczos_bounds
        check(fn(ctx.handle, ctypes.c_void_p(v.data_ptr()), float(tol), int(max_iter), ctypes.byref(lo),
                 ctypes.byref(hi)))
        return lo.value, hi.value


def fermi_level(eigs, weights, nelectron: float, beta: float, smearing: str = "fermi-dirac") -> float:
    """Occupation::find_fermi_level (src/electronic/Occupation.cpp:48-84)."""
    lib = _lib.load()
    e = np.ascontiguousarray(eigs, dtype=np.float64).ravel()
    w = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    ef = ctypes.c_double()
    check(lib.lynx_fermi_level(dptr(e), dptr(w), len(e), float(nelectron), float(beta), _SMEAR[smearing],
                               ctypes.byref(ef)))
    return ef.value


def occupations(eigs, ef: float, beta: float, smearing: str = "fermi-dirac") -> np.ndarray:
    lib = _lib.load()
    e = np.ascontiguousarray(eigs, dtype=np.float64).ravel()
    occ = np.zeros_like(e)
    check(lib.lynx_occupations(dptr(e), len(e), float(ef), float(beta), _SMEAR[smearing], dptr(occ)))
    return occ


def electron_density(ctx: Context, psi, occ, weight: float = 2.0, rho=None, complex_: bool = False):
    """ElectronDensity::compute for one (spin, k-point) block (lynx_electron_density):
    rho (+)= sum_n weight occ[n] |psi_n|^2.  psi: host (Nd, nband) or device (nband, Nd);
    rho: a device tensor of Nd doubles to accumulate into, or None for a new one.  Returns rho
    (a torch CUDA tensor)."""
    torch = _torch()
    ctx.sync_stream()
    a = _DeviceArgs(ctx, psi, complex_)
    occ = np.ascontiguousarray(occ, dtype=np.float64)
    if occ.shape[0] != a.ncol:
        raise ValueError("one occupation per orbital column is needed")
    acc = rho is not None
    if rho is None:
        rho = torch.empty(ctx.nd, dtype=torch.float64, device=f"cuda:{ctx.device}")
    check(ctx.lib.lynx_electron_density(ctx.handle, ctypes.c_void_p(_dev_ptr(a.t)), a.ncol, ctx.nd, dptr(occ),
                                        float(weight), ctypes.c_void_p(_dev_ptr(rho)), 1 if complex_ else 0,
                                        1 if acc else 0))
    return rho


def randomize_orbitals(ctx: Context, nband: int, seed: int, complex_: bool = False):
    """Device start orbitals as EigenSolver::randomize_psi_gpu draws them (cuRAND default
    generator, uniform (0, 1], seed as given): a torch tensor (nband, Nd), float64 or complex128
    (real and imaginary parts interleaved, as the generator fills them)."""
    torch = _torch()
    ctx.sync_stream()
    t = torch.empty((nband, ctx.nd * (2 if complex_ else 1)), dtype=torch.float64, device=f"cuda:{ctx.device}")
    check(ctx.lib.lynx_randomize_orbitals(ctx.handle, ctypes.c_void_p(t.data_ptr()), int(nband), ctx.nd,
                                          ctypes.c_ulonglong(int(seed)), 1 if complex_ else 0))
    return torch.view_as_complex(t.view(nband, ctx.nd, 2)) if complex_ else t


def randomize_orbitals_all(ctx: Context, nband: int, nspin_local: int, nkpts: int, spin_start: int = 0,
                           complex_: bool = False):
    """Every (spin, k-point) block as EigenSolver::randomize_psi_gpu draws them, one generator
    kept across the blocks (lynx_randomize_orbitals_all): a list of nspin_local * nkpts tensors
    (nband, Nd), float64 or complex128, block i = s * nkpts + k."""
    torch = _torch()
    ctx.sync_stream()
    nsk = nspin_local * nkpts
    w = ctx.nd * (2 if complex_ else 1)
    ts = [torch.empty((nband, w), dtype=torch.float64, device=f"cuda:{ctx.device}") for _ in range(nsk)]
    ptrs = (ctypes.c_void_p * nsk)(*[t.data_ptr() for t in ts])
    check(ctx.lib.lynx_randomize_orbitals_all(ctx.handle, ptrs, int(nspin_local), int(spin_start), int(nkpts),
                                              int(nband), 1 if complex_ else 0))
    if complex_:
        return [torch.view_as_complex(t.view(nband, ctx.nd, 2)) for t in ts]
    return ts


def solve_batch(solvers, psis, Veffs, lambda_cutoffs, eigval_mins, eigval_maxs, cheb_degree: int = 20,
                precision: Optional[str] = None, kpt=False):
    """One CheFSI pass of several independent problems at once (lynx_eigensolver_solve_batch).

    Problem i is solvers[i].solve (or solve_kpt when kpt[i]) on psis[i] with Veffs[i]; the
    problems are the k-points and spins of one cell or the cells of an ensemble, each on its
    own Context.  Every distinct context gets a stream of its own for the call, and the passes
    run concurrently from host threads.  Returns [(psi_out, eig)], in order, as solve does;
    each solver's lambda_cutoff is updated."""
    torch = _torch()
    nb = len(solvers)
    kflags = [bool(k) for k in (kpt if isinstance(kpt, (list, tuple)) else [kpt] * nb)]
    if not (len(psis) == len(Veffs) == len(lambda_cutoffs) == len(eigval_mins) == len(eigval_maxs) ==
            len(kflags) == nb):
        raise ValueError("solve_batch: every per-problem list must have one entry per solver")
    if nb == 0:
        return []
    prec = _PREC[precision or solvers[0].precision]
    args = [_DeviceArgs(sv.ctx, p, k) for sv, p, k in zip(solvers, psis, kflags)]
    vs = [_veff_dev(sv.ctx, V) for sv, V in zip(solvers, Veffs)]
    eigs = [np.zeros(a.ncol) for a in args]
    # inputs were written on the current streams; the passes run on streams of their own
    for dev in {sv.ctx.device for sv in solvers}:
        torch.cuda.current_stream(dev).synchronize()
    streams = {}
    for sv in solvers:
        h = sv.ctx.handle.value
        if h not in streams:
            streams[h] = torch.cuda.Stream(device=sv.ctx.device)
            sv.ctx.set_stream(streams[h])
    P = ctypes.c_void_p * nb
    I = ctypes.c_int * nb
    D = ctypes.c_double * nb
    ctxs = P(*[sv.ctx.handle.value for sv in solvers])
    psi_p = P(*[_dev_ptr(a.t) for a in args])
    eig_p = P(*[e.ctypes.data for e in eigs])
    v_p = P(*[v.data_ptr() for v in vs])
    nband = I(*[a.ncol for a in args])
    ld = I(*[sv.ctx.nd for sv in solvers])
    lc = D(*[float(x) for x in lambda_cutoffs])
    lo = D(*[float(x) for x in eigval_mins])
    hi = D(*[float(x) for x in eigval_maxs])
    isk = I(*[1 if k else 0 for k in kflags])
    lc_out = D()
    lib = solvers[0].ctx.lib
    try:
        check(lib.lynx_eigensolver_solve_batch(ctxs, nb, psi_p, eig_p, v_p, nband, ld, lc, lo, hi, isk,
                                               int(cheb_degree), prec, lc_out))
    finally:
        for st in streams.values():
            st.synchronize()
        for sv in solvers:
            sv.ctx.sync_stream()
    out = []
    for i, (sv, a) in enumerate(zip(solvers, args)):
        sv._lambda_cutoff = lc_out[i]
        out.append((a.out(a.t), eigs[i]))
    return out
