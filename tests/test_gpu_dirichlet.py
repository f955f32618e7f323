"""Dirichlet (zero-ghost) directions on the GPU against the reference's own CPU code built with
BCType::Dirichlet (oracle/_ref: FDGrid, HaloExchange, Hamiltonian, EigenSolver compiled
unmodified; src/parallel/HaloExchange.cpp:14-39: non-periodic ghosts stay zero; grid spacing
L / (N - 1) in those directions) and the numpy oracle's restatement.  Mixed boundaries:
Dirichlet in x and z, periodic in y.  Tolerances as for the periodic parity tests: H psi <= 1e-12,
FP64 filter <= 1e-10, FP32 filter <= 2e-5 per column."""
import numpy as np
import pytest

from helpers import rel_err
from lynx_b200 import cell as C
from oracle import chefsi_oracle as O
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dcell():
    from lynx_b200 import solver
    cl, pos = C.diamond_si(1, 20, displace=0.0)
    cl = C.Cell(cl.latvec, (20, 22, 24), True, (1, 0, 1), 12)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=9)
    op = O.Operator(cl.latvec, cl.shape, order=12, orthogonal=True, bc=cl.bc)
    ctx = solver.Context(cl)
    R = ref.RefLynx(cl)
    return dict(cell=cl, V=V, op=op, ctx=ctx, solver=solver, R=R)


def test_dirichlet_stencil_coefficients(dcell):
    mine = dcell["ctx"].stencil_coeffs()
    st = dcell["op"].st
    for k in ("D2x", "D2y", "D2z", "D1x", "D1y", "D1z"):
        np.testing.assert_allclose(mine[k], st[k], rtol=1e-14, atol=1e-14)


def test_dirichlet_hamiltonian(dcell):
    psi = C.random_orbitals(dcell["ctx"].nd, 3, seed=91)
    y_ref = dcell["op"].apply(psi, dcell["V"], 0.3)
    y = dcell["solver"].Hamiltonian(dcell["ctx"], dcell["V"]).apply(psi, shift=0.3)
    assert rel_err(y, y_ref) < 1e-12
    assert rel_err(y, dcell["R"].h_apply(psi, dcell["V"], 0.3)) < 1e-12


def test_dirichlet_filter(dcell):
    X = C.random_orbitals(dcell["ctx"].nd, 4, seed=92)
    lo, hi = -1.5, dcell["ctx"].max_eigval_half_lap + 2.0
    lc = 0.5 * (lo + hi)
    Y_ref = O.chebyshev_filter(dcell["op"], X, dcell["V"], lc, lo, hi, 6)
    es = dcell["solver"].EigenSolver(dcell["ctx"])
    Y = es.chebyshev_filter(X, dcell["V"], lc, lo, hi, 6, precision="fp64")
    assert rel_err(Y, Y_ref) < 1e-10
    Y_cref = dcell["R"].chebyshev_filter(X, dcell["V"], lc, lo, hi, 6)
    assert rel_err(Y, Y_cref) < 1e-10
    Ym = es.chebyshev_filter(X, dcell["V"], lc, lo, hi, 6, precision="mixed")
    for j in range(4):
        assert rel_err(Ym[:, j], Y_cref[:, j]) < 2e-5


def test_dirichlet_pass_matches_reference(dcell):
    """One FP64 CheFSI pass with Dirichlet x and z against the reference's EigenSolver::solve."""
    X = C.random_orbitals(dcell["ctx"].nd, 10, seed=93)
    lo, hi = dcell["R"].lanczos(dcell["V"])
    lc = 0.5 * (lo + hi)
    _, eig_r = dcell["R"].solve(X, dcell["V"], lc, lo, hi, 12)
    _, eig = dcell["solver"].EigenSolver(dcell["ctx"], "fp64").solve(X, dcell["V"], lc, lo, hi, 12)
    assert np.abs(eig - eig_r).max() < 1e-9
