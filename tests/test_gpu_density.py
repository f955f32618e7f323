"""Electron density on the GPU against the reference's own ElectronDensity::compute
(src/electronic/ElectronDensity.cpp:55-172, compiled into oracle/_ref), for one spin channel:
  * lynx_electron_density on given orbitals (real, and complex at a k-point of weight 0.25);
  * lynx_eigensolver_solve_density: a CheFSI pass, the Fermi level of its own Ritz values, and
    the density of the new orbitals -- in the mixed pass accumulated by the tensor-core rotation
    from the FP64 orbitals it writes (with several 128-state tiles and a ragged last one), in the
    FP64 pass by the separate kernel.  Checked against the reference density of the orbitals the
    pass returned, with the occupations of the reference's Occupation (Fermi-Dirac).
FP64 sums in another order than the reference's: 1e-13 of the largest density value."""
import ctypes

import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import _lib
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sys8(synth_psp8):
    from lynx_b200 import solver
    cl, pos, V = si8_small()
    ctx = solver.Context(cl)
    ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
    R = ref.RefLynx(cl, pos, synth_psp8)
    return dict(cl=cl, pos=pos, V=V, ctx=ctx, R=R, solver=solver)


@pytest.mark.parametrize("kpt", [False, True])
def test_density_matches_reference(sys8, kpt):
    s = sys8
    psi = C.random_orbitals(s["ctx"].nd, 7, seed=31, complex_=kpt)
    occ = np.array([1.0, 1.0, 0.8, 0.5, 0.2, 1e-17, 0.0])
    wk = 0.25 if kpt else 1.0
    rho = s["solver"].electron_density(s["ctx"], psi, occ, weight=2.0 * wk, complex_=kpt).cpu().numpy()
    rho_ref = s["R"].density(psi, occ, complex_=kpt, wk=wk)
    assert np.abs(rho - rho_ref).max() <= 1e-13 * np.abs(rho_ref).max()
    # accumulation over blocks (spins / k-points)
    import torch
    r2 = torch.from_numpy(rho).cuda()
    s["solver"].electron_density(s["ctx"], psi, occ, weight=2.0 * wk, rho=r2, complex_=kpt)
    assert np.abs(r2.cpu().numpy() - 2 * rho_ref).max() <= 2e-13 * np.abs(rho_ref).max()


@pytest.mark.parametrize("prec,nband", [("mixed", 150), ("fp64", 40)])
def test_solve_density_matches_reference(sys8, prec, nband):
    import torch
    s = sys8
    ctx, R = s["ctx"], s["R"]
    lo, hi = R.lanczos(s["V"])
    lc = 0.5 * (lo + hi)
    psi = torch.from_numpy(np.ascontiguousarray(C.random_orbitals(ctx.nd, nband, seed=33).T)).cuda()
    V = torch.from_numpy(s["V"]).cuda()
    rho = torch.zeros(ctx.nd, dtype=torch.float64, device="cuda")
    eig = np.zeros(nband)
    lco, ef = ctypes.c_double(), ctypes.c_double()
    nel, beta = 32.0, 1000.0  # Si8: 4 valence electrons per atom; 0.001 Ha Fermi-Dirac smearing
    ctx.sync_stream()
    _lib.check(ctx.lib.lynx_eigensolver_solve_density(
        ctx.handle, ctypes.c_void_p(psi.data_ptr()), _lib.dptr(eig), ctypes.c_void_p(V.data_ptr()), nband, ctx.nd,
        lc, lo, hi, 10, _lib.PREC_MIXED if prec == "mixed" else _lib.PREC_FP64, ctypes.byref(lco), nel, beta,
        _lib.SMEAR_FERMI_DIRAC, 2.0, ctypes.c_void_p(rho.data_ptr()), ctypes.byref(ef)))
    torch.cuda.synchronize()
    ef_ref = ref.fermi_level(eig, 2.0 * np.ones(nband), nel, beta)
    assert abs(ef.value - ef_ref) < 1e-12
    occ = np.array([ref.smearing(e - ef_ref, beta) for e in eig])
    rho_ref = R.density(psi.cpu().numpy().T, occ)
    assert np.abs(rho.cpu().numpy() - rho_ref).max() <= 1e-13 * np.abs(rho_ref).max()
    assert abs(rho.sum().item() * ctx.dV - nel) < 1e-6 * nel  # the orbitals are dV-orthonormal
