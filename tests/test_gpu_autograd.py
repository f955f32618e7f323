"""Adjoints behind torch.autograd.Function (lynx_b200.autograd), on the GPU:
* H psi: the loss L = <w, H(psi, V)> is linear in psi and in V, so a central difference along a
  random direction equals the gradient's directional derivative up to rounding (1e-9 relative);
* E_nl: quadratic in psi, so the central difference is again exact up to rounding;
* E_nl and <w, H psi> in the atom positions, with the projector tables rebuilt at every
  displaced position: the gradients (for E_nl minus the nonlocal force of
  src/physics/Forces.cpp:509-797) against the GPU central differences at R +- h, h = 1e-3 Bohr.
  The force formula projects the FD gradient of psi (summation by parts) while the difference
  moves the sampled projector, so they agree to the grid discretisation of the projector
  gradient: 1e-3 relative, as for the CPU oracle's pin;
* the kinetic + nonlocal energy in a diagonal strain: its gradient (the stress diagonal) against
  central differences of the energy in strained cells."""
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
    assert torch.isfinite(pos.grad).all()


def test_nonlocal_energy_position_gradient_central_difference(synth_psp8):
    """The position gradient against E_nl(R +- h) on the GPU with rebuilt projector tables."""
    import torch
    from lynx_b200 import solver
    from lynx_b200.autograd import nonlocal_energy
    psp = P.read_psp8(synth_psp8)
    cl, pos = C.diamond_si(1, 24, displace=0.05, seed=7)
    ctx = solver.Context(cl)
    rng = np.random.default_rng(3)
    pts = cl.grid_points_cart()
    psi_h = np.zeros((3, ctx.nd))  # smooth band-limited orbitals (low-frequency plane-wave mixtures)
    for n in range(3):
        for _ in range(6):
            kv = 2 * np.pi * rng.integers(-2, 3, size=3) / cl.lengths
            psi_h[n] += rng.normal() * np.cos(pts @ kv + rng.uniform(0, 2 * np.pi))
    psi = _dev(torch, psi_h)
    occ = np.array([1.0, 0.7, 0.2])
    R = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    E = nonlocal_energy(ctx, psi, R, occ, 2.0, psp)
    E.backward()
    grad = R.grad.numpy()
    h = 1e-3
    for atom, dim in ((0, 0), (3, 1), (5, 2), (6, 0)):
        e = []
        for sgn in (1, -1):
            p2 = torch.tensor(pos, dtype=torch.float64)
            p2[atom, dim] += sgn * h
            e.append(float(nonlocal_energy(ctx, psi, p2, occ, 2.0, psp)))
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd) > 0.1 and abs(grad[atom, dim] - fd) <= 1e-3 * abs(fd), (atom, dim, grad[atom, dim], fd)
    ctx.close()


def test_hamiltonian_position_adjoint_central_difference(synth_psp8):
    """The position adjoint of H psi: for L = <w, H(R) psi> the gradient in the atom positions
    against L(R +- h) on the GPU with the projector tables rebuilt at every displaced position
    (h = 1e-3 Bohr).  The adjoint projects FD gradients (summation by parts), so it agrees with the
    difference to the grid discretisation of the projector gradient: 1e-3 relative."""
    import torch
    from lynx_b200 import solver
    from lynx_b200.autograd import hamiltonian_apply
    psp = P.read_psp8(synth_psp8)
    cl, pos = C.diamond_si(1, 24, displace=0.05, seed=11)
    ctx = solver.Context(cl)
    rng = np.random.default_rng(5)
    pts = cl.grid_points_cart()

    def smooth(n):
        out = np.zeros((n, ctx.nd))
        for i in range(n):
            for _ in range(6):
                kv = 2 * np.pi * rng.integers(-2, 3, size=3) / cl.lengths
                out[i] += rng.normal() * np.cos(pts @ kv + rng.uniform(0, 2 * np.pi))
        return out

    psi = _dev(torch, smooth(3))
    w = _dev(torch, smooth(3))
    V = _dev(torch, np.zeros(ctx.nd))
    R = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    L = (w * hamiltonian_apply(ctx, psi, V, R, psp)).sum()
    L.backward()
    grad = R.grad.numpy()
    h = 1e-3
    checked = 0
    for atom in range(len(pos)):
        for dim in range(3):
            e = []
            for sgn in (1, -1):
                p2 = torch.tensor(pos, dtype=torch.float64)
                p2[atom, dim] += sgn * h
                with torch.no_grad():
                    e.append(float((w * hamiltonian_apply(ctx, psi, V, p2, psp)).sum()))
            fd = (e[0] - e[1]) / (2 * h)
            if abs(fd) < 0.05:
                continue
            checked += 1
            assert abs(grad[atom, dim] - fd) <= 1e-3 * abs(fd), (atom, dim, grad[atom, dim], fd)
            if checked >= 4:
                break
        if checked >= 4:
            break
    assert checked >= 4
    ctx.close()


def test_strain_energy_gradient_central_difference(synth_psp8):
    """The strain adjoint: d(E_k + E_nl)/d strain[a] (the diagonal of the GPU kinetic + nonlocal
    stress, in the strained cell) against central differences of the energy at strain +- h
    (h = 1e-4), the projector tables rebuilt in each strained cell.  The kinetic part is exact up
    to the difference's O(h^2); the nonlocal part agrees to the grid discretisation of the
    summation by parts with the FD gradient: 1e-3 relative."""
    import torch
    from lynx_b200.autograd import strain_energy
    psp = P.read_psp8(synth_psp8)
    cl, pos = C.diamond_si(1, 24, displace=0.05, seed=11)
    rng = np.random.default_rng(9)
    pts = cl.grid_points_cart()
    psi_h = np.zeros((3, cl.nd))
    for n in range(3):
        for _ in range(6):
            kv = 2 * np.pi * rng.integers(-2, 3, size=3) / cl.lengths
            psi_h[n] += rng.normal() * np.cos(pts @ kv + rng.uniform(0, 2 * np.pi))
    psi = _dev(torch, psi_h)
    occ = np.array([1.0, 0.6, 0.25])
    eps = torch.tensor([0.004, -0.006, 0.002], dtype=torch.float64, requires_grad=True)
    E = strain_energy(cl, pos, psp, psi, occ, eps)
    E.backward()
    grad = eps.grad.numpy()
    h = 1e-4
    for a in range(3):
        e = []
        for sgn in (1, -1):
            e2 = eps.detach().clone()
            e2[a] += sgn * h
            e.append(float(strain_energy(cl, pos, psp, psi, occ, e2)))
        fd = (e[0] - e[1]) / (2 * h)
        assert abs(fd) > 1.0 and abs(grad[a] - fd) <= 1e-3 * abs(fd), (a, grad[a], fd)
