"""Batched CheFSI passes (lynx_eigensolver_solve_batch) against one-at-a-time solves.

The batch runs each problem's pass from its own host thread on its own stream; the
arithmetic of every problem is unchanged, so the results must be bitwise equal to the
sequential solves of the same problems (the stencil launch-shape autotuner is switched off on
both sides, since concurrent timing could pick another shape).  The problems mix complex
k-point problems of the primitive FCC Si cell with real Gamma-point problems of strained Si8
cells on different grids and band counts.
"""
import numpy as np
import pytest

from lynx_b200 import _lib
from lynx_b200 import cell as C
from lynx_b200 import ensemble as E
from lynx_b200 import pseudo as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problems(synth_psp8):
    from lynx_b200 import solver
    psp = P.read_psp8(synth_psp8)
    probs = E.kpoint_problems(psp, kgrid=(2, 2, 2), grid=16, nband=12)[:4]
    probs += E.strained_ensemble(psp, n_cells=3, grids=(20, 22, 24), nband=16, seed=5)
    ctxs, solvers, bounds = [], [], []
    for i, pb in enumerate(probs):
        ctx = solver.Context(pb.cell)
        ctx.set_option(_lib.OPT_AUTOTUNE, 0)
        ctx.set_nonlocal(pb.tables)
        if pb.complex:
            ctx.set_kpoint(pb.kcart)
        es = solver.EigenSolver(ctx, "fp64")
        lo, hi = es.lanczos_bounds(pb.veff, kpt=pb.complex)
        ctxs.append(ctx)
        solvers.append(es)
        bounds.append((0.5 * (lo + hi), lo, hi))
    psi0 = [C.random_orbitals(c.nd, pb.nband, seed=100 + i, complex_=pb.complex)
            for i, (c, pb) in enumerate(zip(ctxs, probs))]
    return dict(probs=probs, ctxs=ctxs, solvers=solvers, bounds=bounds, psi0=psi0, solver=solver)


def _sequential(s, precision, degree):
    out = []
    for es, pb, b, p in zip(s["solvers"], s["probs"], s["bounds"], s["psi0"]):
        fn = es.solve_kpt if pb.complex else es.solve
        out.append(fn(p, pb.veff, b[0], b[1], b[2], degree, precision=precision))
    return out


def _batched(s, precision, degree, order=None):
    idx = list(range(len(s["probs"]))) if order is None else order
    pb = [s["probs"][i] for i in idx]
    res = s["solver"].solve_batch([s["solvers"][i] for i in idx], [s["psi0"][i] for i in idx],
                                  [q.veff for q in pb], [s["bounds"][i][0] for i in idx],
                                  [s["bounds"][i][1] for i in idx], [s["bounds"][i][2] for i in idx],
                                  degree, precision=precision, kpt=[q.complex for q in pb])
    back = [None] * len(s["probs"])
    for j, i in enumerate(idx):
        back[i] = res[j]
    return back


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_bitwise_equals_sequential(problems, precision):
    seq = _sequential(problems, precision, 12)
    bat = _batched(problems, precision, 12)
    for (p1, e1), (p2, e2) in zip(seq, bat):
        assert np.array_equal(e1, e2)
        assert np.array_equal(p1, p2)


def test_batch_lambda_cutoff_and_order(problems):
    """Results do not depend on the order of the problems in the batch; each solver's
    lambda_cutoff becomes its last Ritz value + 0.1 (EigenSolver.cpp:817)."""
    a = _batched(problems, "fp64", 10)
    b = _batched(problems, "fp64", 10, order=list(reversed(range(len(problems["probs"])))))
    for (p1, e1), (p2, e2), es in zip(a, b, problems["solvers"]):
        assert np.array_equal(e1, e2) and np.array_equal(p1, p2)
        assert es.lambda_cutoff() == pytest.approx(e2[-1] + 0.1, abs=1e-12)


def test_batch_shared_context_runs_in_order(problems):
    """Two problems on one context share its work buffers, so they run one after the other
    on one thread; each gives what a call of its own gives."""
    s = problems
    es, pb, b = s["solvers"][0], s["probs"][0], s["bounds"][0]
    p_a, _ = es.solve_kpt(s["psi0"][0], pb.veff, b[0], b[1], b[2], 8)
    p_b, e_b = es.solve_kpt(s["psi0"][0] * 0.5, pb.veff, b[0], b[1], b[2], 8)
    res = s["solver"].solve_batch([es, es], [s["psi0"][0], s["psi0"][0] * 0.5], [pb.veff, pb.veff],
                                  [b[0], b[0]], [b[1], b[1]], [b[2], b[2]], 8, kpt=True)
    assert np.array_equal(res[0][0], p_a)
    assert np.array_equal(res[1][0], p_b) and np.array_equal(res[1][1], e_b)


def test_batch_reports_failing_problem(problems):
    """A problem with an invalid argument fails the batch with that problem's index."""
    s = problems
    es, pb, b = s["solvers"][-1], s["probs"][-1], s["bounds"][-1]
    bad_veff = np.zeros(7)
    with pytest.raises(ValueError):
        s["solver"].solve_batch([es], [s["psi0"][-1]], [bad_veff], [b[0]], [b[1]], [b[2]], 8)
    good = s["solvers"][-2]
    p_ok, e_ok = good.solve(s["psi0"][-2], s["probs"][-2].veff, *s["bounds"][-2], 8)
    lc_good = good.lambda_cutoff()
    with pytest.raises(_lib.LynxError, match="batch problem 1"):
        # lambda_cutoff above eigmax: rejected before any work
        s["solver"].solve_batch([good, es], [s["psi0"][-2], s["psi0"][-1]],
                                [s["probs"][-2].veff, pb.veff], [s["bounds"][-2][0], b[2] + 1.0],
                                [s["bounds"][-2][1], b[1]], [s["bounds"][-2][2], b[2]], 8)
    assert good.lambda_cutoff() == lc_good


@pytest.fixture(scope="module")
def mixed_grids(synth_psp8):
    """Problems on grids whose stencil launches need different amounts of dynamic shared memory,
    with the launch-shape autotuner on (it times shapes on first use, concurrently here)."""
    from lynx_b200 import solver
    psp = P.read_psp8(synth_psp8)
    probs = E.kpoint_problems(psp, kgrid=(2, 2, 2), grid=20, nband=16)[:2]
    probs += E.strained_ensemble(psp, n_cells=5, grids=(24, 28, 32), nband=24, seed=11)
    solvers, bounds, psi0 = [], [], []
    for i, pb in enumerate(probs):
        ctx = solver.Context(pb.cell)
        ctx.set_nonlocal(pb.tables)
        if pb.complex:
            ctx.set_kpoint(pb.kcart)
        es = solver.EigenSolver(ctx, "mixed")
        lo, hi = es.lanczos_bounds(pb.veff, kpt=pb.complex)
        solvers.append(es)
        bounds.append((0.5 * (lo + hi), lo, hi))
        psi0.append(C.random_orbitals(ctx.nd, pb.nband, seed=200 + i, complex_=pb.complex))
    return dict(probs=probs, solvers=solvers, bounds=bounds, psi0=psi0, solver=solver)


def test_batch_autotuned_mixed_grids(mixed_grids):
    """Concurrent first launches on different grids (the shared-memory cap of a kernel is one
    value per process) complete; once the shapes are chosen, batched equals sequential bitwise."""
    s = mixed_grids
    first = _batched(s, "mixed", 10)
    seq = _sequential(s, "mixed", 10)
    for (p1, e1), (p2, e2) in zip(first, seq):
        # launch shapes timed under load may differ from those timed alone: FP32 filter rounding
        assert np.abs(e1 - e2).max() < 1e-5
    again = _batched(s, "mixed", 10)
    for (p1, e1), (p2, e2) in zip(again, seq):
        assert np.array_equal(e1, e2) and np.array_equal(p1, p2)
