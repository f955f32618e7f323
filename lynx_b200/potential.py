"""Effective potential of an SCF iteration on the GPU (the reference's EffectivePotential,
XCFunctional and PoissonSolver for one spin channel): GGA-PBE exchange-correlation, the AAR
Poisson solve and V_eff = V_xc + phi, through lynx_xc_gga_pbe / lynx_poisson_solve /
lynx_effective_potential.  Fields are FP64 with Nd entries (x fastest); host arrays are copied to
the context's device, torch CUDA tensors are used in place.  Results are torch CUDA tensors."""
from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np

from ._lib import check
from .solver import Context, _dev_ptr, _torch


def _field(ctx: Context, x, name: str):
    torch = _torch()
    if x is None:
        return None
    if isinstance(x, torch.Tensor):
        t = x.to(device=f"cuda:{ctx.device}", dtype=torch.float64).contiguous().reshape(-1)
    else:
        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64).reshape(-1)).to(f"cuda:{ctx.device}")
    if t.numel() != ctx.nd:
        raise ValueError(f"{name} must have Nd = {ctx.nd} entries")
    return t


def _ptr(t):
    return ctypes.c_void_p(_dev_ptr(t)) if t is not None else None


def _empty(ctx: Context):
    torch = _torch()
    return torch.empty(ctx.nd, dtype=torch.float64, device=f"cuda:{ctx.device}")


class XCResult(NamedTuple):
    vxc: object
    exc: object
    dxcdgrho: object


def xc_gga_pbe(ctx: Context, rho, rho_core=None, want_dxcdgrho: bool = False) -> XCResult:
    """XCFunctional::evaluate for GGA_PBE (src/xc/XCFunctional.cpp:193-273): exc, vxc (with the
    GGA divergence term) and, on request, Dxcdgrho = 2 d(rho eps)/d sigma."""
    ctx.sync_stream()
    r = _field(ctx, rho, "rho")
    c = _field(ctx, rho_core, "rho_core")
    vxc, exc = _empty(ctx), _empty(ctx)
    dxc = _empty(ctx) if want_dxcdgrho else None
    check(ctx.lib.lynx_xc_gga_pbe(ctx.handle, _ptr(r), _ptr(c), _ptr(vxc), _ptr(exc), _ptr(dxc)))
    return XCResult(vxc, exc, dxc)


class PoissonSolver:
    """PoissonSolver (src/solvers/PoissonSolver.hpp:35-70): AAR with the reference's parameters
    (m = 7, p = 6, omega = beta = 0.6, Jacobi preconditioner) on the context's grid."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def solve(self, rhs, phi=None, tol: float = 1e-8, max_iter: int = 3000):
        """-Lap phi = rhs from the start phi (zeros when None); returns (phi, iterations)."""
        ctx = self.ctx
        ctx.sync_stream()
        b = _field(ctx, rhs, "rhs")
        x = _field(ctx, phi, "phi")
        x = x.clone() if x is not None else _torch().zeros(ctx.nd, dtype=_torch().float64, device=f"cuda:{ctx.device}")
        it = ctypes.c_int(0)
        check(ctx.lib.lynx_poisson_solve(ctx.handle, _ptr(b), _ptr(x), float(tol), int(max_iter), ctypes.byref(it)))
        return x, it.value


class VeffResult(NamedTuple):
    veff: object
    vxc: object
    exc: object
    phi: object
    poisson_iters: int


class EffectivePotential:
    """EffectivePotential::compute for one spin channel (src/physics/EffectivePotential.cpp:73-177):
    V_eff = V_xc(rho [+ rho_core]) + phi, -Lap phi = 4 pi (rho + rho_b) with the mean removed.
    The electrostatic potential is kept between calls as the next solve's start, as the
    reference keeps it in VeffArrays."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.phi = None

    def compute(self, rho, rho_b=None, rho_core=None, poisson_tol: float = 1e-8) -> VeffResult:
        ctx = self.ctx
        ctx.sync_stream()
        r = _field(ctx, rho, "rho")
        b = _field(ctx, rho_b, "rho_b")
        c = _field(ctx, rho_core, "rho_core")
        if self.phi is None:
            self.phi = _torch().zeros(ctx.nd, dtype=_torch().float64, device=f"cuda:{ctx.device}")
        veff, vxc, exc = _empty(ctx), _empty(ctx), _empty(ctx)
        it = ctypes.c_int(0)
        check(ctx.lib.lynx_effective_potential(ctx.handle, _ptr(r), _ptr(b), _ptr(c), float(poisson_tol), _ptr(veff),
                                               _ptr(vxc), _ptr(exc), _ptr(self.phi), ctypes.byref(it)))
        return VeffResult(veff, vxc, exc, self.phi.clone(), it.value)
