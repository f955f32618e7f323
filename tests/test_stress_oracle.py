"""CPU pin of the stress oracle (src/physics/Stress.cpp:1041-1784, restated in
oracle/chefsi_oracle.py:kinetic_nonlocal_stress) against finite differences of the energies
under a homogeneous strain of an orthogonal cell along axis a: grid points, atoms and cell
stretch by (1 + eps), orbital values on the grid points stay, and psi is rescaled by
(1 + eps)^-1/2 so that its norm is kept.

* Kinetic: E_k(eps) = 1/2 occfac sum_n g_n sum_i |grad_FD psi_n|^2 dV with the FD gradient
  of the strained grid.  dE_k/deps = stress_k[aa] exactly (up to the O(eps^2) of the central
  difference): bar 1e-7 relative.
* Nonlocal: E_nl(eps) = occfac sum_n g_n sum Gamma alpha^2 with the projector tables rebuilt in
  the strained cell.  dE_nl/deps = stress_nl[aa] up to the grid discretisation of the summation
  by parts with the FD gradient (as for the forces): bar 1e-3 relative.
"""
import numpy as np

from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import chefsi_oracle as O


def _tab(t):
    return dict(img_atom=t.img_atom, img_ndc=t.img_ndc, img_shift=t.img_shift, img_coords=t.img_coords,
                gpos=t.gpos, chi=t.chi, gamma=t.gamma, nproj=int(t.atom_nproj[0]))


def _orbitals(cl, nband, seed):
    """Smooth band-limited orbitals (random low-frequency plane-wave mixtures)."""
    rng = np.random.default_rng(seed)
    pts = cl.grid_points_cart()
    psi = np.zeros((cl.nd, nband))
    for n in range(nband):
        for _ in range(6):
            kv = 2 * np.pi * rng.integers(-2, 3, size=3) / cl.lengths
            psi[:, n] += rng.normal() * np.cos(pts @ kv + rng.uniform(0, 2 * np.pi))
    return psi


def _strained(cl, pos, axis, eps):
    f = np.ones(3)
    f[axis] += eps
    cl2 = C.Cell(cl.latvec * f[None, :], cl.shape, True, tuple(cl.bc), cl.fd_order)
    return cl2, pos * f[None, :]


def test_stress_matches_strain_derivatives(synth_psp8):
    cl, pos = C.diamond_si(1, 24, displace=0.05, seed=11)
    psp = P.read_psp8(synth_psp8)
    psi = _orbitals(cl, 3, 5)
    occ = np.array([1.0, 0.6, 0.25])
    st = O.stencil(cl.latvec, cl.shape, 12, True)
    tab = _tab(P.nonlocal_tables(cl, pos, psp))
    sk, snl, e0 = O.kinetic_nonlocal_stress(psi, occ, tab, st, cl, st["dV"], occfac=2.0)
    assert e0 != 0.0
    assert np.all(sk[[0, 3, 5]] < 0)
    h = 1e-4
    for axis, v in ((0, 0), (1, 3), (2, 5)):
        ek, en = [], []
        for sgn in (1, -1):
            cl2, p2 = _strained(cl, pos, axis, sgn * h)
            st2 = O.stencil(cl2.latvec, cl2.shape, 12, True)
            psi2 = psi * (1.0 + sgn * h) ** -0.5
            G = O.cartesian_gradients(psi2, cl2, st2)
            ek.append(0.5 * 2.0 * st2["dV"] * float(sum(np.sum(occ * np.sum(g * g, axis=0)) for g in G)))
            t2 = _tab(P.nonlocal_tables(cl2, p2, psp))
            _, _, e = O.kinetic_nonlocal_stress(psi2, occ, t2, st2, cl2, st2["dV"], occfac=2.0)
            en.append(e)
        dk = (ek[0] - ek[1]) / (2 * h)
        dn = (en[0] - en[1]) / (2 * h)
        assert abs(sk[v] - dk) <= 1e-7 * abs(dk), (axis, sk[v], dk)
        assert abs(snl[v] - dn) <= 1e-3 * max(1.0, abs(dn)), (axis, snl[v], dn)
