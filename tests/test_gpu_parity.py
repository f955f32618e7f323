"""GPU parity: the CUDA path (through the C ABI) against the reference CPU hot path.

The checker is oracle/_ref/libref_lynx.so: the reference LYNX EigenSolver /
Hamiltonian / NonlocalProjector sources compiled unmodified.  Both sides get the
same seeded inputs and the same projector tables.

Tolerances (written per test):
  * FP64 operators (H psi, Vnl psi, filter): max |diff| / max |ref| <= 1e-12 (stencil)
    and <= 1e-10 (degree-m filter, where the recurrence amplifies rounding);
  * FP64 CheFSI pass: Ritz values within 1e-9 Ha, Ritz subspaces within 1e-7;
  * FP32 filter (mixed precision): relative 2e-5 per filter block.
"""
import numpy as np
import pytest

from helpers import rel_err, si8_small, subspace_distance
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system(synth_psp8):
    import torch
    from lynx_b200 import solver
    cl, pos, V = si8_small()
    R = ref.RefLynx(cl, pos, synth_psp8)
    ctx = solver.Context(cl)
    tab = P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8))
    ctx.set_nonlocal(tab)
    return dict(cell=cl, pos=pos, V=V, R=R, ctx=ctx, solver=solver, torch=torch, synth_psp8=synth_psp8)


def test_grid_matches_reference(system):
    R, ctx = system["R"], system["ctx"]
    assert ctx.nd == R.nd
    assert abs(ctx.dV - R.dV) < 1e-15
    st = R.stencil()
    mine = ctx.stencil_coeffs()
    for k in ("D2x", "D2y", "D2z", "D1x", "D1y", "D1z"):
        np.testing.assert_allclose(mine[k], st[k], rtol=1e-14, atol=1e-14)
    assert abs(ctx.max_eigval_half_lap - st["max_eigval"]) < 1e-12


@pytest.mark.parametrize("ncol,shift", [(1, 0.0), (5, 0.0), (3, 0.37)])
def test_hamiltonian_apply_real(system, ncol, shift):
    s = system
    psi = C.random_orbitals(s["ctx"].nd, ncol, seed=11 + ncol)
    y_ref = s["R"].h_apply(psi, s["V"], shift)
    y = s["solver"].Hamiltonian(s["ctx"], s["V"]).apply(psi, shift=shift)
    assert rel_err(y, y_ref) < 1e-12


def test_hamiltonian_apply_device_tensor(system):
    s = system
    torch = s["torch"]
    psi = C.random_orbitals(s["ctx"].nd, 4, seed=5)
    y_ref = s["R"].h_apply(psi, s["V"])
    t = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    y = s["solver"].Hamiltonian(s["ctx"]).apply(t, Veff=torch.from_numpy(s["V"]).cuda())
    assert y.shape == t.shape and y.is_cuda
    assert rel_err(y.cpu().numpy().T, y_ref) < 1e-12


def test_hamiltonian_apply_kpt(system):
    s = system
    cl = s["cell"]
    k = np.array([0.11, -0.23, 0.31]) * 2 * np.pi / cl.lengths
    psi = C.random_orbitals(s["ctx"].nd, 3, seed=7, complex_=True)
    y_ref = s["R"].h_apply_kpt(psi, s["V"], k, 0.1)
    s["ctx"].set_kpoint(k)
    y = s["solver"].Hamiltonian(s["ctx"], s["V"]).apply_kpt(psi, shift=0.1)
    assert rel_err(y, y_ref) < 1e-12


def test_nonlocal_apply(system):
    s = system
    psi = C.random_orbitals(s["ctx"].nd, 6, seed=9)
    h0 = C.random_orbitals(s["ctx"].nd, 6, seed=10)
    y_ref = s["R"].nl_apply(psi, h0)
    y = s["solver"].NonlocalProjector(s["ctx"]).apply(psi, np.array(h0))
    assert rel_err(y, y_ref) < 1e-12


def _bounds(s):
    lo, hi = s["R"].lanczos(s["V"])
    return lo, hi, 0.5 * (lo + hi)


def test_lanczos_bounds(system):
    s = system
    lo_r, hi_r = s["R"].lanczos(s["V"])
    lo, hi = s["solver"].EigenSolver(s["ctx"]).lanczos_bounds(s["V"])
    assert abs(lo - lo_r) < 1e-6 * max(1.0, abs(lo_r))
    assert abs(hi - hi_r) < 1e-6 * abs(hi_r)


@pytest.mark.parametrize("degree", [1, 2, 7])
def test_chebyshev_filter_fp64(system, degree):
    s = system
    lo, hi, lc = _bounds(s)
    X = C.random_orbitals(s["ctx"].nd, 6, seed=21)
    Y_ref = s["R"].chebyshev_filter(X, s["V"], lc, lo, hi, degree)
    Y = s["solver"].EigenSolver(s["ctx"]).chebyshev_filter(X, s["V"], lc, lo, hi, degree, precision="fp64")
    assert rel_err(Y, Y_ref) < 1e-10


def test_chebyshev_filter_mixed(system):
    s = system
    lo, hi, lc = _bounds(s)
    X = C.random_orbitals(s["ctx"].nd, 6, seed=21)
    Y_ref = s["R"].chebyshev_filter(X, s["V"], lc, lo, hi, 12)
    Y = s["solver"].EigenSolver(s["ctx"]).chebyshev_filter(X, s["V"], lc, lo, hi, 12, precision="mixed")
    for j in range(6):  # per column, relative to the column's own scale
        assert rel_err(Y[:, j], Y_ref[:, j]) < 2e-5


def test_chebyshev_filter_kpt(system):
    s = system
    cl = s["cell"]
    k = np.array([0.25, 0.0, -0.25]) * 2 * np.pi / cl.lengths
    lo, hi = s["R"].lanczos(s["V"], kpt=k)
    lc = 0.5 * (lo + hi)
    X = C.random_orbitals(s["ctx"].nd, 4, seed=33, complex_=True)
    Y_ref = s["R"].chebyshev_filter_kpt(X, s["V"], lc, lo, hi, 8, k)
    s["ctx"].set_kpoint(k)
    Y = s["solver"].EigenSolver(s["ctx"]).chebyshev_filter(X, s["V"], lc, lo, hi, 8, precision="fp64", kpt=True)
    assert rel_err(Y, Y_ref) < 1e-10


def test_solve_fp64_matches_reference(system):
    s = system
    lo, hi, lc = _bounds(s)
    N = 16
    psi0 = C.random_orbitals(s["ctx"].nd, N, seed=41)
    psi_r, eig_r = s["R"].solve(psi0, s["V"], lc, lo, hi, 20)
    es = s["solver"].EigenSolver(s["ctx"], "fp64")
    psi, eig = es.solve(psi0, s["V"], lc, lo, hi, 20)
    assert np.all(np.diff(eig) >= -1e-12)
    assert np.abs(eig - eig_r).max() < 1e-9
    assert abs(es.lambda_cutoff() - (eig[-1] + 0.1)) < 1e-12
    assert subspace_distance(psi, psi_r) < 1e-7


def test_solve_kpt_fp64_matches_reference(system):
    s = system
    cl = s["cell"]
    k = np.array([0.25, 0.25, 0.0]) * 2 * np.pi / cl.lengths
    lo, hi = s["R"].lanczos(s["V"], kpt=k)
    lc = 0.5 * (lo + hi)
    N = 10
    psi0 = C.random_orbitals(s["ctx"].nd, N, seed=43, complex_=True)
    psi_r, eig_r = s["R"].solve_kpt(psi0, s["V"], lc, lo, hi, 16, k)
    s["ctx"].set_kpoint(k)
    psi, eig = s["solver"].EigenSolver(s["ctx"], "fp64").solve_kpt(psi0, s["V"], lc, lo, hi, 16)
    assert np.abs(eig - eig_r).max() < 1e-9
    assert subspace_distance(psi, psi_r) < 1e-7


def test_scf_like_convergence_mixed_vs_fp64(system):
    """Repeated CheFSI passes at fixed V (the SCF inner loop): the mixed-precision
    path converges to the same occupied Ritz values as the FP64 path (<= 1e-6 Ha)."""
    s = system
    lo, hi, lc0 = _bounds(s)
    N = 16
    out = {}
    for prec in ("fp64", "mixed"):
        es = s["solver"].EigenSolver(s["ctx"], prec)
        psi = C.random_orbitals(s["ctx"].nd, N, seed=77)
        lc, emin = lc0, lo
        for it in range(12):
            psi, eig = es.solve(psi, s["V"], lc, emin, hi, 20)
            lc = es.lambda_cutoff()
            emin = eig[0]
        out[prec] = eig
    nocc = 12
    assert np.abs(out["mixed"][:nocc] - out["fp64"][:nocc]).max() < 1e-6


@pytest.fixture(scope="module")
def odd_system(synth_psp8):
    """Odd grid dimensions: FP64 blocks need padded rows; the caller layout uses the fallback kernel."""
    from lynx_b200 import solver
    cl, pos, V = si8_small(grid=(15, 17, 19))
    R = ref.RefLynx(cl, pos, synth_psp8)
    ctx = solver.Context(cl)
    ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
    return dict(cell=cl, pos=pos, V=V, R=R, ctx=ctx, solver=solver)


def test_odd_grid_apply_filter_solve(odd_system):
    s = odd_system
    psi = C.random_orbitals(s["ctx"].nd, 3, seed=3)
    assert rel_err(s["solver"].Hamiltonian(s["ctx"], s["V"]).apply(psi), s["R"].h_apply(psi, s["V"])) < 1e-12
    lo, hi = s["R"].lanczos(s["V"])
    lc = 0.5 * (lo + hi)
    es = s["solver"].EigenSolver(s["ctx"])
    Y = es.chebyshev_filter(psi, s["V"], lc, lo, hi, 5, precision="fp64")
    assert rel_err(Y, s["R"].chebyshev_filter(psi, s["V"], lc, lo, hi, 5)) < 1e-10
    Ym = es.chebyshev_filter(psi, s["V"], lc, lo, hi, 5, precision="mixed")
    assert rel_err(Ym, s["R"].chebyshev_filter(psi, s["V"], lc, lo, hi, 5)) < 2e-5
    psi0 = C.random_orbitals(s["ctx"].nd, 8, seed=4)
    _, eig_r = s["R"].solve(psi0, s["V"], lc, lo, hi, 12)
    _, eig = es.solve(psi0, s["V"], lc, lo, hi, 12, precision="fp64")
    assert np.abs(eig - eig_r).max() < 1e-9


@pytest.mark.parametrize("n", [40])
def test_free_particle_known_answer(n):
    """tests/unit/test_Hamiltonian.cpp:39-112: on a 2*pi cube with V = 0, H sin(x) = 0.5 sin(x)
    (FD12, N = 40, error < 1e-6); a constant orbital gives V*psi."""
    from lynx_b200 import solver
    L = 2 * np.pi
    cl = C.Cell(np.eye(3) * L, (n, n, n))
    ctx = solver.Context(cl)
    x = np.arange(n) * L / n
    psi = np.tile(np.sin(x), n * n)
    H = solver.Hamiltonian(ctx)
    y = H.apply(psi, np.zeros(ctx.nd))
    assert np.abs(y - 0.5 * psi).max() < 1e-6
    V = 0.3 + 0.1 * np.cos(np.tile(x, n * n))
    y2 = H.apply(np.ones(ctx.nd), V)
    assert np.abs(y2 - V).max() < 1e-10


@pytest.mark.parametrize("nstates", [150])
def test_mixed_pass_tensor_core_gram(system, nstates):
    """Mixed precision real pass (FP32 filter, exact int8-slice tensor-core Gram products with
    FP64 split-K reduction, FP64 subspace algebra) against the FP64 pass from the same start:
    more than one 128-state output tile, a ragged last tile.  Ritz values agree to 2e-5 Ha
    (FP32 filter rounding dominates), the spectrum stays ordered and both passes span the
    same subspace."""
    s = system
    lo, hi, lc = _bounds(s)
    psi0 = C.random_orbitals(s["ctx"].nd, nstates, seed=151)
    out = {}
    for prec in ("fp64", "mixed"):
        es = s["solver"].EigenSolver(s["ctx"], prec)
        out[prec] = es.solve(psi0, s["V"], lc, lo, hi, 10)
    eig64, eigm = out["fp64"][1], out["mixed"][1]
    assert np.all(np.diff(eigm) >= -1e-9)
    assert np.abs(eigm - eig64).max() < 2e-5
    assert subspace_distance(out["mixed"][0], out["fp64"][0]) < 1e-3


def test_fused_nonlocal_and_shapes_bitwise(system):
    """The fused nonlocal term (stencil kernel adds a * chi alpha), with the projections read from
    the full grid or from the compact sphere-point copy the previous step wrote, and every launch
    shape give bitwise the results of the separate-scatter default-shape path (same operations,
    same order)."""
    from lynx_b200 import _lib
    s = system
    lo, hi, lc = _bounds(s)
    X = C.random_orbitals(s["ctx"].nd, 20, seed=91)
    out = {}
    for fuse, tune, compact in ((0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1)):
        ctx = s["solver"].Context(s["cell"])
        ctx.set_nonlocal(P.nonlocal_tables(s["cell"], s["pos"], P.read_psp8(s["synth_psp8"])))
        _lib.check(ctx.lib.lynx_set_option(ctx.handle, _lib.OPT_FUSE_NONLOCAL, fuse))
        _lib.check(ctx.lib.lynx_set_option(ctx.handle, _lib.OPT_AUTOTUNE, tune))
        _lib.check(ctx.lib.lynx_set_option(ctx.handle, _lib.OPT_COMPACT_GATHER, compact))
        es = s["solver"].EigenSolver(ctx)
        for prec in ("fp64", "mixed"):
            out[(fuse, tune, compact, prec)] = es.chebyshev_filter(X, s["V"], lc, lo, hi, 6, precision=prec)
        ctx.close()
    for prec in ("fp64", "mixed"):
        ref_ = out[(0, 0, 0, prec)]
        for key in ((0, 1, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1)):
            assert np.array_equal(out[key + (prec,)], ref_), (key, prec)


def test_fused_nonlocal_wide_rows_bitwise(synth_psp8):
    """A wider grid (36 x 20 x 40) whose z extent recycles every ring stage of the fused stencil
    several times, each stage carrying a different W range: the fused term and its compact copy
    give bitwise the separate-scatter results in both precisions."""
    from lynx_b200 import _lib, solver
    cl, pos, V = si8_small(grid=(36, 20, 40), seed=5)
    X = C.random_orbitals(int(np.prod(cl.shape)), 12, seed=93)
    out = {}
    for fuse, compact in ((0, 0), (1, 0), (1, 1)):
        ctx = solver.Context(cl)
        ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
        _lib.check(ctx.lib.lynx_set_option(ctx.handle, _lib.OPT_FUSE_NONLOCAL, fuse))
        _lib.check(ctx.lib.lynx_set_option(ctx.handle, _lib.OPT_COMPACT_GATHER, compact))
        es = solver.EigenSolver(ctx)
        lo, hi = es.lanczos_bounds(V)
        for prec in ("fp64", "mixed"):
            out[(fuse, compact, prec)] = es.chebyshev_filter(X, V, 0.5 * (lo + hi), lo, hi, 5, precision=prec)
        ctx.close()
    for prec in ("fp64", "mixed"):
        for key in ((1, 0), (1, 1)):
            assert np.array_equal(out[key + (prec,)], out[(0, 0, prec)]), (key, prec)


@pytest.mark.parametrize("block", [0, 64, 37])
def test_host_solve_pipelined_matches_device(system, block):
    """lynx_eigensolver_solve_host copies psi in column blocks on a second stream and filters
    each block as it lands (mixed precision, >= 256 states; default blocks of 128 columns, and
    LYNX_OPT_HOST_COPY_BLOCK 64 and 37): bitwise the device-pointer pass."""
    import ctypes
    from lynx_b200 import _lib
    s = system
    lo, hi, lc = _bounds(s)
    N = 300
    psi0 = C.random_orbitals(s["ctx"].nd, N, seed=201)
    hp = np.asfortranarray(psi0.copy())
    eig_h = np.zeros(N)
    V = np.ascontiguousarray(s["V"], dtype=np.float64)
    lco = ctypes.c_double()
    _lib.check(s["ctx"].lib.lynx_set_option(s["ctx"].handle, _lib.OPT_HOST_COPY_BLOCK, block))
    try:
        _lib.check(s["ctx"].lib.lynx_eigensolver_solve_host(s["ctx"].handle, _lib.dptr(hp), _lib.dptr(eig_h),
                                                           _lib.dptr(V), N, s["ctx"].nd, lc, lo, hi, 8,
                                                           _lib.PREC_MIXED, ctypes.byref(lco)))
    finally:
        _lib.check(s["ctx"].lib.lynx_set_option(s["ctx"].handle, _lib.OPT_HOST_COPY_BLOCK, 0))
    psi_d, eig_d = s["solver"].EigenSolver(s["ctx"], "mixed").solve(psi0, s["V"], lc, lo, hi, 8)
    assert np.array_equal(eig_h, np.asarray(eig_d))
    assert np.array_equal(hp, np.asarray(psi_d))


def test_every_stencil_shape_bitwise(system):
    """Every compiled launch shape of the pipelined stencil and both band splits
    (LYNX_OPT_STENCIL_SHAPE k = 1..8), with the fused nonlocal term: bitwise the default shape's
    filter, both precisions."""
    from lynx_b200 import _lib
    s = system
    lo, hi, lc = _bounds(s)
    X = C.random_orbitals(s["ctx"].nd, 10, seed=95)
    ctx = s["solver"].Context(s["cell"])
    ctx.set_nonlocal(P.nonlocal_tables(s["cell"], s["pos"], P.read_psp8(s["synth_psp8"])))
    es = s["solver"].EigenSolver(ctx)
    out = {}
    for k in range(0, 9):
        _lib.check(ctx.lib.lynx_set_option(ctx.handle, _lib.OPT_STENCIL_SHAPE, k))
        for prec in ("fp64", "mixed"):
            out[(k, prec)] = es.chebyshev_filter(X, s["V"], lc, lo, hi, 4, precision=prec)
    ctx.close()
    for prec in ("fp64", "mixed"):
        for k in range(1, 9):
            assert np.array_equal(out[(k, prec)], out[(0, prec)]), (k, prec)
