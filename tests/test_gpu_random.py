"""Device start orbitals (lynx_randomize_orbitals): the reference's GPU path fills them with
cuRAND's default generator, uniform (0, 1], seeded per (spin, k-point)
(src/solvers/EigenSolver.cu:1199-1228).  The same library call with the same seed gives the
same values; here: determinism, the range, seed sensitivity, the complex layout, and the
moments of a uniform distribution."""
import numpy as np
import pytest

from helpers import si8_small

pytestmark = pytest.mark.gpu


def test_randomize_orbitals():
    import torch
    from lynx_b200 import solver
    cl, _, _ = si8_small()
    ctx = solver.Context(cl)
    seed = 0 * 1000 + 0 * 13 + 1  # spin 0, first k-point, spin_start 0
    a = solver.randomize_orbitals(ctx, 6, seed)
    b = solver.randomize_orbitals(ctx, 6, seed)
    c = solver.randomize_orbitals(ctx, 6, seed + 13)
    torch.cuda.synchronize()
    assert a.shape == (6, ctx.nd) and a.dtype == torch.float64
    assert torch.equal(a, b)
    assert not torch.equal(a, c)
    x = a.cpu().numpy()
    assert x.min() > 0.0 and x.max() <= 1.0
    assert abs(x.mean() - 0.5) < 5e-3 and abs(x.var() - 1.0 / 12.0) < 5e-3
    z = solver.randomize_orbitals(ctx, 3, seed, complex_=True)
    assert z.dtype == torch.complex128 and z.shape == (3, ctx.nd)
    # the complex block is the same stream of doubles, read as interleaved (re, im) pairs
    zr = torch.view_as_real(z).reshape(3, -1)
    assert torch.equal(zr.reshape(-1)[:6 * ctx.nd], a.reshape(-1)[:6 * ctx.nd])
