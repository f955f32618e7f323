"""Device start orbitals (lynx_randomize_orbitals): the reference's GPU path fills them with
cuRAND's default generator, uniform (0, 1], seeded per (spin, k-point)
(src/solvers/EigenSolver.cu:1199-1228).  Here: the reference's call sequence replayed through
the cuRAND library (bitwise), determinism, the range, seed sensitivity, the complex layout, and
the moments of a uniform distribution."""
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


def _curand():
    import ctypes
    import os
    for name in ("libcurand.so", "libcurand.so.10", "/usr/local/cuda/lib64/libcurand.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    torch_lib = os.path.join(os.path.dirname(__import__("torch").__file__), "lib")
    for f in sorted(os.listdir(torch_lib)):
        if f.startswith("libcurand"):
            return ctypes.CDLL(os.path.join(torch_lib, f))
    pytest.skip("libcurand not found")


@pytest.mark.parametrize("is_kpt", [False, True])
def test_randomize_matches_the_reference_call_sequence(is_kpt):
    """EigenSolver::randomize_psi_gpu (src/solvers/EigenSolver.cu:1199-1228) replayed through the
    cuRAND library itself: one generator handle kept across the (spin, k-point) blocks, re-seeded
    per block with (spin_start + s) * 1000 + i * 13 + 1, curandGenerateUniformDouble of Nd * Nband
    doubles (twice that for complex blocks).  lynx_randomize_orbitals_all gives bitwise the same
    blocks; lynx_randomize_orbitals (a fresh generator) gives the first one, and -- re-seeding
    does not rewind the generator -- not the later ones."""
    import ctypes
    import torch
    from lynx_b200 import solver
    cl, _, _ = si8_small()
    ctx = solver.Context(cl)
    cur = _curand()
    gen = ctypes.c_void_p()
    assert cur.curandCreateGenerator(ctypes.byref(gen), 100) == 0  # CURAND_RNG_PSEUDO_DEFAULT
    nspin, nkpts, spin_start, nband = 2, 3, 1, 5
    n = ctx.nd * nband * (2 if is_kpt else 1)
    try:
        refs = []
        for i in range(nspin * nkpts):
            s = i // nkpts
            seed = (spin_start + s) * 1000 + i * 13 + 1
            buf = torch.empty(n, dtype=torch.float64, device="cuda")
            assert cur.curandSetPseudoRandomGeneratorSeed(gen, ctypes.c_ulonglong(seed)) == 0
            assert cur.curandGenerateUniformDouble(gen, ctypes.c_void_p(buf.data_ptr()), ctypes.c_size_t(n)) == 0
            refs.append(buf)
        torch.cuda.synchronize()
        ours = solver.randomize_orbitals_all(ctx, nband, nspin, nkpts, spin_start, complex_=is_kpt)
        torch.cuda.synchronize()
        for i, (o, r) in enumerate(zip(ours, refs)):
            got = torch.view_as_real(o).reshape(-1) if is_kpt else o.reshape(-1)
            assert torch.equal(got, r), i
        first = solver.randomize_orbitals(ctx, nband, spin_start * 1000 + 1, complex_=is_kpt)
        second = solver.randomize_orbitals(ctx, nband, spin_start * 1000 + 13 + 1, complex_=is_kpt)
        torch.cuda.synchronize()
        flat = (lambda t: torch.view_as_real(t).reshape(-1)) if is_kpt else (lambda t: t.reshape(-1))
        assert torch.equal(flat(first), refs[0])
        assert not torch.equal(flat(second), refs[1])
    finally:
        cur.curandDestroyGenerator(gen)
        ctx.close()
