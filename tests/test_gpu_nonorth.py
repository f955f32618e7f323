"""GPU parity on a non-orthogonal cell (primitive FCC Si2, 20^3 grid, FD order 12): the mixed-
derivative Laplacian terms (src/operators/Hamiltonian.cpp:177-267) through the C ABI against the
compiled reference, Gamma point and Bloch k-points, FP64 and FP32 filters.

Tolerances as in test_gpu_parity: H psi <= 1e-12 relative, FP64 filter <= 1e-10, CheFSI Ritz
values <= 1e-9 Ha, FP32 filter <= 2e-5 per column."""
import numpy as np
import pytest

from helpers import rel_err
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fcc(synth_psp8):
    from lynx_b200 import solver
    cl, pos = C.fcc_si_primitive(grid=20)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=5)
    R = ref.RefLynx(cl, pos, synth_psp8)
    ctx = solver.Context(cl)
    ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
    k = np.array([0.25, -0.25, 0.5]) * 2 * np.pi / cl.lengths
    return dict(cell=cl, pos=pos, V=V, R=R, ctx=ctx, solver=solver, k=k)


def test_nonorth_stencil_coefficients(fcc):
    st = fcc["R"].stencil()
    mine = fcc["ctx"].stencil_coeffs()
    for key in ("D2x", "D2y", "D2z", "D1x", "D1y", "D1z", "D2xy", "D2xz", "D2yz"):
        np.testing.assert_allclose(mine[key], st[key], rtol=1e-14, atol=1e-14)
    assert np.abs(st["D2xy"]).max() > 0  # the cell really has mixed terms


def test_nonorth_hamiltonian_real(fcc):
    psi = C.random_orbitals(fcc["ctx"].nd, 4, seed=31)
    y_ref = fcc["R"].h_apply(psi, fcc["V"], 0.2)
    y = fcc["solver"].Hamiltonian(fcc["ctx"], fcc["V"]).apply(psi, shift=0.2)
    assert rel_err(y, y_ref) < 1e-12


def test_nonorth_hamiltonian_kpt(fcc):
    psi = C.random_orbitals(fcc["ctx"].nd, 3, seed=32, complex_=True)
    y_ref = fcc["R"].h_apply_kpt(psi, fcc["V"], fcc["k"], 0.0)
    fcc["ctx"].set_kpoint(fcc["k"])
    y = fcc["solver"].Hamiltonian(fcc["ctx"], fcc["V"]).apply_kpt(psi)
    assert rel_err(y, y_ref) < 1e-12


def test_nonorth_filter_and_solve_kpt(fcc):
    s = fcc
    lo, hi = s["R"].lanczos(s["V"], kpt=s["k"])
    lc = 0.5 * (lo + hi)
    X = C.random_orbitals(s["ctx"].nd, 6, seed=33, complex_=True)
    s["ctx"].set_kpoint(s["k"])
    es = s["solver"].EigenSolver(s["ctx"])
    Y_ref = s["R"].chebyshev_filter_kpt(X, s["V"], lc, lo, hi, 8, s["k"])
    Y = es.chebyshev_filter(X, s["V"], lc, lo, hi, 8, precision="fp64", kpt=True)
    assert rel_err(Y, Y_ref) < 1e-10
    Ym = es.chebyshev_filter(X, s["V"], lc, lo, hi, 8, precision="mixed", kpt=True)
    for j in range(6):
        assert rel_err(Ym[:, j], Y_ref[:, j]) < 2e-5
    psi0 = C.random_orbitals(s["ctx"].nd, 10, seed=34, complex_=True)
    _, eig_r = s["R"].solve_kpt(psi0, s["V"], lc, lo, hi, 12, s["k"])
    _, eig = s["solver"].EigenSolver(s["ctx"], "fp64").solve_kpt(psi0, s["V"], lc, lo, hi, 12)
    assert np.abs(eig - eig_r).max() < 1e-9


def test_nonorth_solve_gamma_mixed_vs_fp64(fcc):
    s = fcc
    lo, hi = s["R"].lanczos(s["V"])
    lc = 0.5 * (lo + hi)
    psi0 = C.random_orbitals(s["ctx"].nd, 12, seed=35)
    _, eig_r = s["R"].solve(psi0, s["V"], lc, lo, hi, 12)
    _, eig = s["solver"].EigenSolver(s["ctx"], "fp64").solve(psi0, s["V"], lc, lo, hi, 12)
    assert np.abs(eig - eig_r).max() < 1e-9
