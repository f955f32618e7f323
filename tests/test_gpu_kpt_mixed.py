"""Mixed-precision k-point CheFSI (complex Bloch orbitals): the FP32 filter and the Gram products
and rotation on the real tensor-core kernels through the planar split [Re Y | Im Y] (2N real
states), complex FP64 subspace algebra.  Against the FP64 k-point pass (itself within 1e-9 Ha of
the reference's EigenSolver::solve_kpt, src/solvers/EigenSolver.cpp:826-842) on the
non-orthogonal primitive FCC Si2 cell and an orthogonal Si8 cell:
  * one pass with the tensor-core products against the same pass with FP64 library products of
    the same FP32 blocks: Ritz values within 1e-8 of the largest (the int8-digit products carry
    about 1e-8 relative error), the same subspace;
  * passes iterated from the same start at fixed V_eff until the FP64 occupied Ritz values stop
    moving: mixed within 1e-6 Ha of FP64."""
import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import _lib
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import ref

pytestmark = pytest.mark.gpu


def _system(kind, psp):
    from lynx_b200 import solver
    if kind == "fcc":
        cl, pos = C.fcc_si_primitive(grid=20)
        nband, nocc = 16, 4
    else:
        cl, pos, _ = si8_small()
        nband, nocc = 24, 16
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=7)
    tab = P.nonlocal_tables(cl, pos, P.read_psp8(psp))
    k = np.array([0.25, -0.125, 0.375]) * 2 * np.pi / cl.lengths
    ctx = solver.Context(cl)
    ctx.set_nonlocal(tab)
    ctx.set_kpoint(k)
    return solver, cl, pos, V, ctx, k, nband, nocc


@pytest.mark.parametrize("kind", ["fcc", "si8"])
def test_tensor_core_products_match_fp64_products(synth_psp8, kind):
    solver, cl, pos, V, ctx, k, nband, nocc = _system(kind, synth_psp8)
    es = solver.EigenSolver(ctx, "mixed")
    lo, hi = es.lanczos_bounds(V, kpt=True)
    lc = 0.5 * (lo + hi)
    psi0 = C.random_orbitals(ctx.nd, nband, seed=41, complex_=True)
    out = {}
    for tc in (1, 0):
        ctx.set_option(_lib.OPT_TC_RAYLEIGH_RITZ, tc)
        out[tc] = es.solve_kpt(psi0.copy(), V, lc, lo, hi, 10)
    ctx.set_option(_lib.OPT_TC_RAYLEIGH_RITZ, 1)
    assert np.abs(out[1][1] - out[0][1]).max() < 1e-8 * np.abs(out[0][1]).max()
    # the orbitals span the same subspace: the singular values of the dV-weighted overlap are 1
    # to the rotation's accuracy (about an FP32 product of depth N, 1e-6 of the column norm)
    a, b = np.asarray(out[1][0]), np.asarray(out[0][0])
    sv = np.linalg.svd(a.conj().T @ b * cl.dV, compute_uv=False)
    assert np.abs(sv - 1).max() < 1e-5
    ctx.close()


@pytest.mark.parametrize("kind", ["fcc", "si8"])
def test_mixed_kpt_converges_to_fp64(synth_psp8, kind):
    solver, cl, pos, V, ctx, k, nband, nocc = _system(kind, synth_psp8)
    R = ref.RefLynx(cl, pos, synth_psp8)
    lo, hi = R.lanczos(V, kpt=k)
    psi0 = C.random_orbitals(ctx.nd, nband, seed=43, complex_=True)
    # first pass: FP64 against the reference
    _, eig_r = R.solve_kpt(psi0, V, 0.5 * (lo + hi), lo, hi, 12, k)
    _, eig_1 = solver.EigenSolver(ctx, "fp64").solve_kpt(psi0.copy(), V, 0.5 * (lo + hi), lo, hi, 12)
    assert np.abs(eig_1 - eig_r).max() < 1e-9

    def run(prec, passes):
        es = solver.EigenSolver(ctx, prec)
        psi, lc, emin = psi0.copy(), 0.5 * (lo + hi), lo
        prev, eig, n = None, None, 0
        for n in range(1, passes + 1):
            psi, eig = es.solve_kpt(psi, V, lc, emin, hi, 12)
            lc, emin = es.lambda_cutoff(), float(eig[0])
            if passes == 40 and prev is not None and np.abs(eig[:nocc] - prev).max() < 1e-10:
                break
            prev = eig[:nocc].copy()
        return eig, n

    res = {}
    res["fp64"], n_passes = run("fp64", 40)
    assert n_passes < 40
    res["mixed"], _ = run("mixed", n_passes)
    assert np.abs(res["mixed"][:nocc] - res["fp64"][:nocc]).max() < 1e-6
    ctx.close()
