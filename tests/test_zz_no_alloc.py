"""lynx_nonlocal_apply_noalloc (fixed device scratch, no allocation) against lynx_nonlocal_apply.

Collected last on purpose: it must pass both alone and after every other GPU test has used
the library in the same process.  Two calls in a row check that nothing carried over in the
shared scratch array changes the second result.
"""
import ctypes

import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P

pytestmark = pytest.mark.gpu


def test_noalloc_nonlocal_matches_allocating_entry(synth_psp8):
    import torch
    from lynx_b200 import _lib, solver
    cl, pos, _ = si8_small()
    ctx = solver.Context(cl)
    ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
    lib = ctx.lib
    results = []
    for ncol, seed in ((7, 1), (40, 2)):  # two calls in a row, different widths
        psi = torch.from_numpy(np.ascontiguousarray(C.random_orbitals(ctx.nd, ncol, seed=seed).T)).cuda()
        h0 = torch.from_numpy(np.ascontiguousarray(C.random_orbitals(ctx.nd, ncol, seed=seed + 10).T)).cuda()
        h_ref, h_new = h0.clone(), h0.clone()
        ctx.sync_stream()
        _lib.check(lib.lynx_nonlocal_apply(ctx.handle, ctypes.c_void_p(psi.data_ptr()),
                                           ctypes.c_void_p(h_ref.data_ptr()), ncol, ctx.nd))
        _lib.check(lib.lynx_nonlocal_apply_noalloc(ctx.handle, ctypes.c_void_p(psi.data_ptr()),
                                                   ctypes.c_void_p(h_new.data_ptr()), ncol, ctx.nd))
        ctx.sync_stream()
        results.append((h_ref.cpu().numpy(), h_new.cpu().numpy()))
    for h_ref, h_new in results:
        # same kernels, same order of summation: bitwise equal
        assert np.array_equal(h_ref, h_new)
        assert np.abs(h_ref).max() > 0


def test_noalloc_rejects_oversize(synth_psp8):
    import torch
    from lynx_b200 import _lib, solver
    cl, pos, _ = si8_small()
    ctx = solver.Context(cl)
    tab = P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8))
    ctx.set_nonlocal(tab)
    nproj = int(np.sum(tab.atom_nproj))
    ncol = (8 << 20) // (8 * nproj) + 64  # alpha just over the 8 MiB scratch
    psi = torch.zeros((ncol, ctx.nd), dtype=torch.float64, device="cuda")  # valid memory all the same
    st = ctx.lib.lynx_nonlocal_apply_noalloc(ctx.handle, ctypes.c_void_p(psi.data_ptr()),
                                             ctypes.c_void_p(psi.data_ptr()), ncol, ctx.nd)
    assert st == _lib.LYNX_ERR_BAD_ARG
    assert b"limit" in ctx.lib.lynx_last_error()
