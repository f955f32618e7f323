"""GPU kinetic and nonlocal stress (lynx_kinetic_nonlocal_stress / _kpt) against the reference's
own Stress::compute_nonlocal_kinetic_cpu (src/physics/Stress.cpp:1041-1784, compiled into
oracle/_ref; before its division by the cell measure) and the numpy oracle (pinned to finite
differences of the energies under strain in test_stress_oracle.py), on the same seeded orbitals
and projector tables: an orthogonal Si8 cell and the non-orthogonal primitive FCC Si2 cell,
Gamma point and a Bloch k-point.  FP64 throughout: every component within 1e-10 of the largest
component of its kind."""
import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import chefsi_oracle as O
from oracle import ref

pytestmark = pytest.mark.gpu


def _tab(t):
    return dict(img_atom=t.img_atom, img_ndc=t.img_ndc, img_shift=t.img_shift, img_coords=t.img_coords,
                gpos=t.gpos, chi=t.chi, gamma=t.gamma, nproj=int(t.atom_nproj[0]))


def _system(kind, synth_psp8):
    if kind == "orth":
        cl, pos, _ = si8_small()
    else:
        cl, pos = C.fcc_si_primitive(grid=18)
    return cl, pos, P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8))


@pytest.mark.parametrize("kind,kpt", [("orth", False), ("orth", True), ("fcc", False), ("fcc", True)])
def test_stress_matches_oracle(synth_psp8, kind, kpt):
    from lynx_b200 import solver
    cl, pos, t = _system(kind, synth_psp8)
    ctx = solver.Context(cl)
    ctx.set_nonlocal(t)
    st = O.stencil(cl.latvec, cl.shape, 12, cl.orthogonal)
    psi = C.random_orbitals(ctx.nd, 5, seed=71, complex_=kpt)
    occ = np.array([1.0, 0.9, 0.6, 0.3, 0.05])
    k = None
    wk = 0.25 if kpt else 1.0
    if kpt:
        k = np.array([0.15, -0.2, 0.3]) * 2 * np.pi / cl.lengths
        ctx.set_kpoint(k)
    sk_ref, snl_ref, _ = O.kinetic_nonlocal_stress(psi, occ, _tab(t), st, cl, st["dV"], occfac=2.0, wk=wk, kpt=k)
    sk, snl = solver.NonlocalProjector(ctx).stress(psi, occ, occfac=2.0, kpt=kpt, wk=wk)
    sk_c, snl_c = ref.RefLynx(cl, pos, synth_psp8).kinetic_nonlocal_stress(psi, occ, kpt=k, wk=wk)
    assert np.abs(sk - sk_c).max() <= 1e-10 * np.abs(sk_c).max()
    assert np.abs(snl - snl_c).max() <= 1e-10 * np.abs(snl_c).max()
    assert np.abs(sk - sk_ref).max() <= 1e-10 * np.abs(sk_ref).max()
    assert np.abs(snl - snl_ref).max() <= 1e-10 * np.abs(snl_ref).max()
    assert np.abs(snl_ref).max() > 0


def test_stress_without_projectors(synth_psp8):
    """Without projector tables the nonlocal part is zero and the kinetic part still comes out."""
    from lynx_b200 import solver
    cl, pos, _ = si8_small()
    ctx = solver.Context(cl)
    st = O.stencil(cl.latvec, cl.shape, 12, True)
    psi = C.random_orbitals(ctx.nd, 3, seed=72)
    occ = np.array([1.0, 0.5, 0.25])
    sk_ref, _, _ = O.kinetic_nonlocal_stress(psi, occ, None, st, cl, st["dV"], occfac=1.0)
    sk, snl = solver.NonlocalProjector(ctx).stress(psi, occ, occfac=1.0)
    assert np.abs(sk - sk_ref).max() <= 1e-10 * np.abs(sk_ref).max()
    assert np.all(snl == 0.0)
