"""Error paths of the C ABI, driven on the host so that no GPU faults or hangs:

* a NaN in V_eff reaches the overlap and projected Hamiltonian: the pass returns
  LYNX_ERR_NONFINITE (the reference's GPU path would carry the NaN on silently,
  src/solvers/EigenSolver.cu:258-259,302-305 ignore cuSOLVER's info);
* a start block with a zero column makes the overlap singular: LYNX_ERR_CHOL_FAIL (the
  reference's CPU path throws, src/solvers/EigenSolver.cpp:633-635);
* the bounded device-side wait is made to run out on an mbarrier that nothing completes
  (lynx_selftest_wait_timeout): LYNX_ERR_TIMEOUT, after which the same context still computes
  H psi exactly as before.
Both precisions are checked where the path differs (FP64 cuBLAS products, tensor-core mixed)."""
import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import _lib
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sys8(synth_psp8):
    from lynx_b200 import solver
    cl, pos, V = si8_small()
    ctx = solver.Context(cl)
    ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
    lo, hi = solver.EigenSolver(ctx).lanczos_bounds(V)
    return dict(ctx=ctx, V=V, lo=lo, hi=hi, solver=solver)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_nan_in_veff_is_nonfinite(sys8, prec):
    s = sys8
    V = s["V"].copy()
    V[1234] = np.nan
    psi = C.random_orbitals(s["ctx"].nd, 8, seed=5)
    es = s["solver"].EigenSolver(s["ctx"], prec)
    with pytest.raises(_lib.LynxError) as ei:
        es.solve(psi, V, 0.5 * (s["lo"] + s["hi"]), s["lo"], s["hi"], 6)
    assert ei.value.status == _lib.LYNX_ERR_NONFINITE


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_rank_deficient_start_block_is_chol_fail(sys8, prec):
    s = sys8
    psi = C.random_orbitals(s["ctx"].nd, 8, seed=6)
    psi[:, 3] = 0.0
    es = s["solver"].EigenSolver(s["ctx"], prec)
    with pytest.raises(_lib.LynxError) as ei:
        es.solve(psi, s["V"], 0.5 * (s["lo"] + s["hi"]), s["lo"], s["hi"], 6)
    assert ei.value.status == _lib.LYNX_ERR_CHOL_FAIL


def test_bounded_wait_times_out_and_context_recovers(sys8):
    s = sys8
    ctx = s["ctx"]
    psi = C.random_orbitals(ctx.nd, 3, seed=7)
    H = s["solver"].Hamiltonian(ctx, s["V"])
    y0 = H.apply(psi)
    rc = ctx.lib.lynx_selftest_wait_timeout(ctx.handle, 4096)
    assert rc == _lib.LYNX_ERR_TIMEOUT
    assert b"wait gave up" in ctx.lib.lynx_last_error()
    assert ctx.lib.lynx_selftest_wait_timeout(ctx.handle, 0) == _lib.LYNX_ERR_BAD_ARG
    y1 = H.apply(psi)  # the error flag was cleared: the context computes as before
    assert np.array_equal(y0, y1)
