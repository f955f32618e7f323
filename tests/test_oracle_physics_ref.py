"""The numpy restatements of the forces, stress and density pinned to the reference's own code:
Forces::compute_nonlocal_cpu (src/physics/Forces.cpp:509-797), Stress::compute_nonlocal_kinetic_cpu
(src/physics/Stress.cpp:1041-1784, before its division by the cell measure) and
ElectronDensity::compute (src/electronic/ElectronDensity.cpp:55-172), compiled unmodified into
oracle/_ref.  Same seeded orbitals, occupations and projector tables on both sides; an
orthogonal Si8 cell and the non-orthogonal primitive FCC Si2 cell, Gamma point and a Bloch
k-point with weight 0.25.  FP64 on both sides: 1e-12 of the largest component."""
import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import chefsi_oracle as O
from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _tab(t):
    return dict(img_atom=t.img_atom, img_ndc=t.img_ndc, img_shift=t.img_shift, img_coords=t.img_coords,
                gpos=t.gpos, chi=t.chi, gamma=t.gamma, nproj=int(t.atom_nproj[0]))


def _system(kind, psp_path):
    if kind == "orth":
        cl, pos, _ = si8_small()
    else:
        cl, pos = C.fcc_si_primitive(grid=18)
    return cl, pos, P.nonlocal_tables(cl, pos, P.read_psp8(psp_path))


@pytest.mark.parametrize("kind,kpt", [("orth", False), ("orth", True), ("fcc", False), ("fcc", True)])
def test_forces_stress_density_match_reference(synth_psp8, kind, kpt):
    cl, pos, t = _system(kind, synth_psp8)
    R = ref.RefLynx(cl, pos, synth_psp8)
    st = O.stencil(cl.latvec, cl.shape, 12, cl.orthogonal)
    psi = C.random_orbitals(R.nd, 5, seed=81, complex_=kpt)
    occ = np.array([1.0, 0.9, 0.6, 0.3, 0.05])
    k = np.array([0.15, -0.2, 0.3]) * 2 * np.pi / cl.lengths if kpt else None
    wk = 0.25 if kpt else 1.0
    f_ref = R.nonlocal_force(psi, occ, kpt=k, wk=wk)
    f, _ = O.nonlocal_force(psi, occ, _tab(t), st, cl.shape, st["dV"], occfac=2.0, wk=wk, kpt=k, lengths=cl.lengths)
    assert np.abs(f_ref).max() > 0
    assert np.abs(f - f_ref).max() <= 1e-12 * np.abs(f_ref).max()
    sk_ref, snl_ref = R.kinetic_nonlocal_stress(psi, occ, kpt=k, wk=wk)
    sk, snl, _ = O.kinetic_nonlocal_stress(psi, occ, _tab(t), st, cl, st["dV"], occfac=2.0, wk=wk, kpt=k)
    assert np.abs(sk - sk_ref).max() <= 1e-12 * np.abs(sk_ref).max()
    assert np.abs(snl - snl_ref).max() <= 1e-12 * np.abs(snl_ref).max()
    rho_ref = R.density(psi, occ, complex_=kpt, wk=wk)
    rho = 2.0 * wk * (np.abs(np.asarray(psi)) ** 2 @ occ)
    assert np.abs(rho - rho_ref).max() <= 1e-13 * np.abs(rho_ref).max()


def test_dirichlet_hamiltonian_matches_reference():
    """The numpy restatement of the Dirichlet ghost rule against the reference's own FDGrid /
    HaloExchange / Hamiltonian built with BCType::Dirichlet in x and z (src/core/types.hpp:14,
    src/parallel/HaloExchange.cpp:14-39): spacing L / (N - 1), zero ghosts."""
    from helpers import rel_err
    cl, pos = C.diamond_si(1, 20, displace=0.0)
    cl = C.Cell(cl.latvec, (20, 22, 24), True, (1, 0, 1), 12)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=9)
    op = O.Operator(cl.latvec, cl.shape, order=12, orthogonal=True, bc=cl.bc)
    R = ref.RefLynx(cl)
    assert abs(R.dV - cl.dV) < 1e-15
    psi = C.random_orbitals(R.nd, 3, seed=91)
    assert rel_err(R.h_apply(psi, V, 0.3), op.apply(psi, V, 0.3)) < 1e-13
