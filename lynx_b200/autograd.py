"""Differentiable operators for PyTorch (torch.autograd.Function), on top of the C ABI.

* ``hamiltonian_apply(ctx, psi, veff, positions=None, psp=None)``: y = H psi with H = -0.5 Lap +
  Veff + Vnl (real, Gamma point).  H is symmetric on the grid (symmetric FD stencil, diagonal
  Veff, Vnl = dV chi Gamma chi^T), so the adjoint with respect to the orbitals is H itself,
  grad_psi = H grad_y, and with respect to the potential grad_Veff = sum_n grad_y_n * psi_n.
  With atom positions (and ``psp`` to rebuild the tables there) the positions are an input too:
  for L = sum_n <g_n, Vnl psi_n> = (1/dV) sum_n a(g_n)^T Gamma a(psi_n), a(x) = dV chi^T x,
  dL/dR = (1/dV) sum_n sum_p Gamma_p [b(g_n) a(psi_n) + a(g_n) b(psi_n)]_p with b = da/dR, the
  projection of the FD gradient used by the nonlocal forces.  By the polarisation identity
  a(u)b(v) + a(v)b(u) = (a(u+v)b(u+v) - a(u-v)b(u-v)) / 2, that is two calls of the force kernel
  (lynx_nonlocal_force, F(x) = -2 sum_n sum_p Gamma_p a(x_n) b(x_n) with unit occupations):
  grad_R = (F(psi - g) - F(psi + g)) / (4 dV).
* ``nonlocal_energy(ctx, psi, positions, occ, occfac, psp)``: E_nl = occfac sum_n f_n sum_p
  Gamma_p alpha_{p,n}^2 (alpha = dV chi^T psi_n); grad_psi_n = 2 occfac f_n dV (Vnl psi_n)
  (d alpha / d psi = dV chi, and Vnl psi = chi Gamma alpha), and grad_positions = -F with F the
  nonlocal forces of lynx_nonlocal_force (the formula of the reference's
  Forces::compute_nonlocal, src/physics/Forces.cpp:509-797).  With a pseudopotential ``psp``
  the forward pass rebuilds the context's projector tables at ``positions`` (what the
  reference's NonlocalProjector::setup does for new atom positions), so the energy is a
  function of the positions; without one, the context's current tables are used and must
  belong to ``positions``.  The position gradient is along the lattice directions (Cartesian
  for orthogonal cells).
* ``strain_energy(cell, positions, psp, psi, occ, strain, occfac)``: the kinetic + nonlocal
  band energy under a homogeneous diagonal strain of an orthogonal cell (grid, atoms and cell
  stretch by 1 + strain[a] along axis a; the orbitals keep their grid values, rescaled to keep
  their norm), differentiable in the strain: E = E_k + E_nl with E_k = 1/2 occfac sum_n f_n
  dV |D psi_n|^2 (D the FD gradient: minus half the trace of the kinetic stress) and E_nl from
  the projector tables rebuilt in the strained cell; dE/dstrain[a] = (stress_k[aa] +
  stress_nl[aa]) / (1 + strain[a]) with the stress of lynx_kinetic_nonlocal_stress in the
  strained cell (before the division by the cell measure; the formula of the reference's
  Stress::compute_nonlocal_kinetic, src/physics/Stress.cpp:1041-1784).

Orbitals are torch CUDA tensors of shape (ncol, Nd), float64 (the layout lynx_b200.solver takes
without copies); the computation runs in liblynxb200.so.
"""
from __future__ import annotations

import numpy as np


def _torch():
    import torch
    return torch


def _make_fns():
    torch = _torch()
    from . import solver

    class HamiltonianApply(torch.autograd.Function):
        @staticmethod
        def forward(fctx, psi, veff, positions, ctx, psp):
            if psp is not None and positions is not None:
                from . import pseudo
                R = positions.detach().cpu().numpy().astype(np.float64)
                ctx.set_nonlocal(pseudo.nonlocal_tables(ctx.cell, R, psp))
            fctx.ctx = ctx
            fctx.save_for_backward(psi, veff)
            fctx.pos_like = positions
            return solver.Hamiltonian(ctx).apply(psi.contiguous(), Veff=veff.contiguous())

        @staticmethod
        def backward(fctx, grad_y):
            psi, veff = fctx.saved_tensors
            g = grad_y.contiguous()
            grad_psi = solver.Hamiltonian(fctx.ctx).apply(g, Veff=veff.contiguous()) if fctx.needs_input_grad[0] else None
            grad_v = (g * psi).sum(0) if fctx.needs_input_grad[1] else None
            grad_pos = None
            if fctx.needs_input_grad[2]:
                ones = np.ones(psi.shape[0])
                nl = solver.NonlocalProjector(fctx.ctx)
                fm, _ = nl.force((psi - g).contiguous(), ones, occfac=1.0)
                fp, _ = nl.force((psi + g).contiguous(), ones, occfac=1.0)
                pos = fctx.pos_like
                grad_pos = torch.as_tensor((np.asarray(fm) - np.asarray(fp)) / (4.0 * fctx.ctx.dV),
                                           dtype=pos.dtype, device=pos.device).reshape(pos.shape)
            return grad_psi, grad_v, grad_pos, None, None

    class NonlocalEnergy(torch.autograd.Function):
        @staticmethod
        def forward(fctx, psi, positions, ctx, occ, occfac, psp):
            if psp is not None:
                from . import pseudo
                R = positions.detach().cpu().numpy().astype(np.float64)
                ctx.set_nonlocal(pseudo.nonlocal_tables(ctx.cell, R, psp))
            occ = np.asarray(occ, dtype=np.float64)
            f, e = solver.NonlocalProjector(ctx).force(psi.contiguous(), occ, occfac=occfac)
            fctx.ctx = ctx
            fctx.occ = occ
            fctx.occfac = occfac
            fctx.save_for_backward(psi)
            fctx.force = torch.as_tensor(f, dtype=positions.dtype, device=positions.device)
            return torch.tensor(e, dtype=psi.dtype, device=psi.device)

        @staticmethod
        def backward(fctx, grad_e):
            (psi,) = fctx.saved_tensors
            grad_psi = grad_pos = None
            if fctx.needs_input_grad[0]:
                vnl = solver.NonlocalProjector(fctx.ctx).apply(psi.contiguous(), torch.zeros_like(psi))
                w = torch.as_tensor(2.0 * fctx.occfac * fctx.ctx.dV * fctx.occ, dtype=psi.dtype,
                                    device=psi.device)[:, None]
                grad_psi = grad_e * w * vnl
            if fctx.needs_input_grad[1]:
                grad_pos = -grad_e.to(device=fctx.force.device, dtype=fctx.force.dtype) * fctx.force
            return grad_psi, grad_pos, None, None, None, None

    class StrainEnergy(torch.autograd.Function):
        @staticmethod
        def forward(fctx, strain, cell, positions, psp, psi, occ, occfac):
            from . import pseudo
            from .cell import Cell
            f = 1.0 + strain.detach().cpu().numpy().astype(np.float64).reshape(3)
            cl2 = Cell(np.asarray(cell.latvec) * f[None, :], cell.shape, True, tuple(cell.bc), cell.fd_order)
            ctx2 = solver.Context(cl2, device=psi.device.index or 0)
            try:
                ctx2.set_nonlocal(pseudo.nonlocal_tables(cl2, np.asarray(positions, dtype=np.float64) * f[None, :], psp))
                psi2 = (psi * float(np.prod(f)) ** -0.5).contiguous()
                occ = np.asarray(occ, dtype=np.float64)
                nl = solver.NonlocalProjector(ctx2)
                sk, snl = nl.stress(psi2, occ, occfac=occfac)
                _, enl = nl.force(psi2, occ, occfac=occfac)
            finally:
                ctx2.close()
            # the stress is the derivative in a strain of the strained cell; one more strain d of it
            # is a change of (1 + strain[a]) (1 + d): d/dstrain[a] = stress[aa] / (1 + strain[a])
            fctx.grad = torch.tensor([(sk[0] + snl[0]) / f[0], (sk[3] + snl[3]) / f[1], (sk[5] + snl[5]) / f[2]],
                                     dtype=strain.dtype, device=strain.device)
            e = -0.5 * (sk[0] + sk[3] + sk[5]) + enl
            return torch.tensor(e, dtype=strain.dtype, device=strain.device)

        @staticmethod
        def backward(fctx, grad_e):
            return grad_e * fctx.grad, None, None, None, None, None, None

    return HamiltonianApply, NonlocalEnergy, StrainEnergy


_FNS = None


def _fns():
    global _FNS
    if _FNS is None:
        _FNS = _make_fns()
    return _FNS


def hamiltonian_apply(ctx, psi, veff, positions=None, psp=None):
    """y = H psi, differentiable in psi, veff and (when given) the atom positions; with ``psp`` the
    projector tables are rebuilt at ``positions`` first (see the module docstring)."""
    return _fns()[0].apply(psi, veff, positions, ctx, psp)


def nonlocal_energy(ctx, psi, positions, occ, occfac: float = 2.0, psp=None):
    """E_nl of the orbitals psi, differentiable in psi and in the atom positions (with ``psp``,
    a lynx_b200.pseudo.Psp8, the projector tables are rebuilt at ``positions`` first)."""
    return _fns()[1].apply(psi, positions, ctx, occ, occfac, psp)


def strain_energy(cell, positions, psp, psi, occ, strain, occfac: float = 2.0):
    """Kinetic + nonlocal band energy of psi in the cell stretched by 1 + strain[a] along each axis
    (orthogonal cells), differentiable in ``strain`` (a torch tensor of 3 values); the gradient is
    the diagonal of the kinetic + nonlocal stress (see the module docstring)."""
    if not cell.orthogonal:
        raise ValueError("strain_energy takes orthogonal cells (diagonal strain)")
    return _fns()[2].apply(strain, cell, positions, psp, psi, occ, occfac)
