"""Adjoints behind torch.autograd.Function (lynx_b200.autograd), on the GPU:
* H psi: the loss L = <w, H(psi, V)> is linear in psi and in V, so a central difference along a
  random direction equals the gradient's directional derivative up to rounding (1e-9 relative);
* E_nl: quadratic in psi, so the central difference is again exact up to rounding; the
  position gradient is minus the nonlocal force."""
import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(synth_psp8):
    import torch
    from lynx_b200 import solver
    cl, pos, V = si8_small()
    ctx = solver.Context(cl)
    ctx.set_nonlocal(P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8)))
    return dict(torch=torch, ctx=ctx, cl=cl, pos=pos, V=V)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_hamiltonian_adjoint(setup):
    torch, ctx = setup["torch"], setup["ctx"]
    from lynx_b200.autograd import hamiltonian_apply
    nd = ctx.nd
    psi = _dev(torch, C.random_orbitals(nd, 3, seed=71).T).requires_grad_(True)
    V = _dev(torch, setup["V"]).requires_grad_(True)
    w = _dev(torch, C.random_orbitals(nd, 3, seed=72).T)
    L = (w * hamiltonian_apply(ctx, psi, V)).sum()
    L.backward()
    dpsi = _dev(torch, C.random_orbitals(nd, 3, seed=73).T)
    dV = _dev(torch, np.random.default_rng(74).normal(size=nd))
    eps = 1e-3
    with torch.no_grad():
        def loss(p, v):
            return float((w * hamiltonian_apply(ctx, p, v)).sum())
        fd_psi = (loss(psi + eps * dpsi, V) - loss(psi - eps * dpsi, V)) / (2 * eps)
        fd_v = (loss(psi, V + eps * dV) - loss(psi, V - eps * dV)) / (2 * eps)
    assert abs(float((psi.grad * dpsi).sum()) - fd_psi) <= 1e-9 * max(1.0, abs(fd_psi))
    assert abs(float((V.grad * dV).sum()) - fd_v) <= 1e-9 * max(1.0, abs(fd_v))


def test_nonlocal_energy_gradients(setup):
    torch, ctx = setup["torch"], setup["ctx"]
    from lynx_b200 import solver
    from lynx_b200.autograd import nonlocal_energy
    nd = ctx.nd
    occ = np.array([1.0, 0.6, 0.25])
    psi = _dev(torch, C.random_orbitals(nd, 3, seed=81).T).requires_grad_(True)
    pos = torch.tensor(setup["pos"], dtype=torch.float64, requires_grad=True)
    E = nonlocal_energy(ctx, psi, pos, occ, 2.0)
    E.backward()
    d = _dev(torch, C.random_orbitals(nd, 3, seed=82).T)
    eps = 1e-3
    with torch.no_grad():
        ep = float(nonlocal_energy(ctx, psi + eps * d, pos, occ, 2.0))
        em = float(nonlocal_energy(ctx, psi - eps * d, pos, occ, 2.0))
    fd = (ep - em) / (2 * eps)
    assert abs(float((psi.grad * d).sum()) - fd) <= 1e-9 * max(1.0, abs(fd))
    f, _ = solver.NonlocalProjector(ctx).force(psi.detach(), occ, occfac=2.0)
    assert np.allclose(pos.grad.numpy(), -f, rtol=0, atol=1e-14 * max(1.0, np.abs(f).max()))
