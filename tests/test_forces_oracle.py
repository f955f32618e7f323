"""CPU pin of the nonlocal-force oracle: on an orthogonal cell the force formula of
src/physics/Forces.cpp:509-797 (projections of the FD gradient of psi) equals minus the central
finite difference (h = 1e-3 Bohr) of the nonlocal energy E_nl(R) = occfac sum_n f_n sum Gamma
alpha(R)^2 with the projectors rebuilt at the displaced atom.  The two differ by the grid
discretisation of the projector gradient (summation by parts with the FD gradient; a few 1e-4
relative at h = 0.43 Bohr), so the bar is 1e-3 relative: it pins signs and factors."""
import numpy as np

from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import chefsi_oracle as O


def _tab(t):
    return dict(img_atom=t.img_atom, img_ndc=t.img_ndc, img_shift=t.img_shift, gpos=t.gpos, chi=t.chi,
                gamma=t.gamma, nproj=int(t.atom_nproj[0]))


def test_nonlocal_force_matches_energy_derivative(synth_psp8):
    cl, pos = C.diamond_si(1, 24, displace=0.05, seed=7)
    psp = P.read_psp8(synth_psp8)
    st = O.stencil(cl.latvec, cl.shape, 12, True)
    rng = np.random.default_rng(3)
    nd = int(np.prod(cl.shape))
    # smooth band-limited orbitals (random low-frequency plane-wave mixtures)
    pts = cl.grid_points_cart()
    psi = np.zeros((nd, 3))
    for n in range(3):
        for _ in range(6):
            kv = 2 * np.pi * rng.integers(-2, 3, size=3) / cl.lengths
            psi[:, n] += rng.normal() * np.cos(pts @ kv + rng.uniform(0, 2 * np.pi))
    occ = np.array([1.0, 0.7, 0.2])
    tab = _tab(P.nonlocal_tables(cl, pos, psp))
    f, e0 = O.nonlocal_force(psi, occ, tab, st, cl.shape, st["dV"], occfac=2.0)
    assert e0 != 0.0
    h = 1e-3
    for atom, dim in ((0, 0), (3, 1), (5, 2)):
        ep, em = [], []
        for sgn, lst in ((1, ep), (-1, em)):
            p2 = pos.copy()
            p2[atom, dim] += sgn * h
            t2 = _tab(P.nonlocal_tables(cl, p2, psp))
            _, e = O.nonlocal_force(psi, occ, t2, st, cl.shape, st["dV"], occfac=2.0)
            lst.append(e)
        fd = -(ep[0] - em[0]) / (2 * h)
        assert abs(f[atom, dim] - fd) <= 1e-3 * max(1.0, abs(fd)), (atom, dim, f[atom, dim], fd)
