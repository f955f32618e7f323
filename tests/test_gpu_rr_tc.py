"""Direct tests of the tensor-core Rayleigh-Ritz kernels of the mixed-precision pass, through the
C ABI (lynx_gram_mixed -> gram_i8_kernel, lynx_rotate_mixed -> rot_i8_kernel), element by element
against FP64 products of the same FP32 data (cuBLAS DGEMM through torch on the same device; its
rounding, ~1e-16 relative, is far below the bars).

The reference computes these products in FP64 (src/solvers/EigenSolver.cu:195-233 overlap and
projection, :312-329 rotation).  Bars:
  * Gram: max_ij |dMs_ij| / sqrt(Ms_ii Ms_jj) <= 1e-7 (upper triangle), and the same for Hs
    with sqrt(Ms_ii |hy_j|^2 scale);
  * rotation: per state j, the relative 2-norm error ||dpsi_j|| / ||psi_j|| <= 2e-6 and
    max_r |dpsi_rj| / max_r |psi_rj| <= 3e-6, and no worse than 4x an FP32 GEMM of the same
    FP32 data (cuBLAS SGEMM, TF32 off): the rotation is meant to be as accurate as an FP32
    product of depth N.
Cases: the Si216 workload's shape (729 088 rows, 520 states: five 128-state tiles with a ragged
last one, K split into chunks), 129 states (a one-state ragged tile), and a K extent that is not
a multiple of the 128-row K step.  Column scales span four decades, as the filtered blocks do."""
import ctypes

import numpy as np
import pytest

from lynx_b200 import _lib
from lynx_b200 import cell as C

pytestmark = pytest.mark.gpu

CASES = [(729088, 520), (200_004, 129), (65_540, 160)]


@pytest.fixture(scope="module")
def ctx():
    from lynx_b200 import solver
    cl = C.Cell(np.eye(3) * 10.0, (20, 20, 20))
    c = solver.Context(cl)
    yield c
    c.close()


def _blocks(torch, rows, n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    scale = 10.0 ** (4.0 * torch.rand(n, generator=g, device="cuda", dtype=torch.float64) - 2.0)
    Y = (torch.randn(n, rows, generator=g, device="cuda", dtype=torch.float64) * scale[:, None]).float()
    # HY: a smooth mix of Y's rows plus independent noise (the projected operator is not diagonal)
    HY = (0.7 * Y.double() + 0.3 * torch.randn(n, rows, generator=g, device="cuda", dtype=torch.float64)
          * scale[:, None]).float()
    return Y.contiguous(), HY.contiguous()


@pytest.mark.parametrize("rows,n", CASES)
def test_gram_mixed_matches_fp64(ctx, rows, n):
    import torch
    Y, HY = _blocks(torch, rows, n, seed=rows + n)
    Ms = torch.zeros(n, n, device="cuda", dtype=torch.float64)
    Hs = torch.zeros(n, n, device="cuda", dtype=torch.float64)
    scale = 0.037
    torch.cuda.synchronize()
    _lib.check(ctx.lib.lynx_gram_mixed(ctx.handle, ctypes.c_void_p(Y.data_ptr()), ctypes.c_void_p(HY.data_ptr()),
                                       rows, rows, n, scale, ctypes.c_void_p(Ms.data_ptr()),
                                       ctypes.c_void_p(Hs.data_ptr())))
    Y64, H64 = Y.double(), HY.double()
    # column-major N x N results: element (i, j) at [j][i] of the row-major torch view
    Ms_ref = (scale * (Y64 @ Y64.T)).T
    Hs_ref = (scale * (Y64 @ H64.T)).T
    d = torch.sqrt(torch.diagonal(Ms_ref))
    dh = torch.sqrt(scale * (H64 * H64).sum(1))
    upper = torch.triu(torch.ones(n, n, dtype=torch.bool, device="cuda"))  # (i <= j) in column-major
    em = ((Ms - Ms_ref).abs() / (d[None, :] * d[:, None]))[upper.T].max().item()
    eh = ((Hs - Hs_ref).abs() / (dh[:, None] * d[None, :])).max().item()
    assert em <= 1e-7, em
    assert eh <= 1e-7, eh


@pytest.mark.parametrize("rows,n", CASES)
def test_rotate_mixed_matches_fp64(ctx, rows, n):
    import torch
    Y, _ = _blocks(torch, rows, n, seed=3 * rows + n)
    Y64 = Y.double()
    scale = 0.037
    Ms = scale * (Y64 @ Y64.T)  # symmetric: the same in either storage order
    # W = R^-1 Q as the pass forms it: R^T R = Ms (upper R), Q orthogonal
    R = torch.linalg.cholesky(Ms).T
    g = torch.Generator(device="cuda").manual_seed(rows)
    Q, _ = torch.linalg.qr(torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64))
    W = torch.linalg.solve_triangular(R, Q, upper=True)
    Wc = W.T.contiguous()  # column-major storage of W
    psi = torch.zeros(n, rows, device="cuda", dtype=torch.float64)
    torch.cuda.synchronize()
    _lib.check(ctx.lib.lynx_rotate_mixed(ctx.handle, ctypes.c_void_p(Y.data_ptr()), rows, rows,
                                         ctypes.c_void_p(Ms.data_ptr()), ctypes.c_void_p(Wc.data_ptr()), n,
                                         ctypes.c_void_p(psi.data_ptr()), rows))
    ref = (Y64.T @ W).T  # psi_ref[j] = sum_i W[i, j] y_i

    def errs(p):
        d = p - ref
        return ((d.norm(dim=1) / ref.norm(dim=1)).max().item(),
                (d.abs().max(1).values / ref.abs().max(1).values).max().item())

    e2, emax = errs(psi)
    torch.backends.cuda.matmul.allow_tf32 = False
    f2, _ = errs((Y.T @ W.float()).T.double())
    assert e2 <= 2e-6 and emax <= 3e-6, (e2, emax)
    assert e2 <= 4.0 * f2, (e2, f2)


def test_gram_mixed_flags_nan(ctx):
    import torch
    Y, HY = _blocks(torch, 4096, 8, seed=5)
    HY[3, 100] = float("nan")
    Ms = torch.zeros(8, 8, device="cuda", dtype=torch.float64)
    Hs = torch.zeros_like(Ms)
    torch.cuda.synchronize()
    rc = ctx.lib.lynx_gram_mixed(ctx.handle, ctypes.c_void_p(Y.data_ptr()), ctypes.c_void_p(HY.data_ptr()), 4096,
                                 4096, 8, 1.0, ctypes.c_void_p(Ms.data_ptr()), ctypes.c_void_p(Hs.data_ptr()))
    assert rc == _lib.LYNX_ERR_NONFINITE
