"""GPU nonlocal forces and energy (lynx_nonlocal_force / _kpt) against the reference's own
Forces::compute_nonlocal_cpu (src/physics/Forces.cpp:509-797, compiled into oracle/_ref) and the
numpy oracle (for the energy, which that routine does not return), on the same seeded orbitals
and projector tables.  FP64: forces within 1e-10 relative to the largest component, energies
within 1e-12 relative."""
import numpy as np
import pytest

from helpers import si8_small
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P
from oracle import chefsi_oracle as O
from oracle import ref

pytestmark = pytest.mark.gpu


def _tab(t):
    return dict(img_atom=t.img_atom, img_ndc=t.img_ndc, img_shift=t.img_shift, gpos=t.gpos, chi=t.chi,
                gamma=t.gamma, nproj=int(t.atom_nproj[0]))


@pytest.mark.parametrize("kpt", [False, True])
def test_nonlocal_force_matches_oracle(synth_psp8, kpt):
    from lynx_b200 import solver
    cl, pos, _ = si8_small()
    t = P.nonlocal_tables(cl, pos, P.read_psp8(synth_psp8))
    ctx = solver.Context(cl)
    ctx.set_nonlocal(t)
    st = O.stencil(cl.latvec, cl.shape, 12, True)
    psi = C.random_orbitals(ctx.nd, 7, seed=61, complex_=kpt)
    occ = np.linspace(1.0, 0.1, 7)
    k = None
    wk = 0.5 if kpt else 1.0
    if kpt:
        k = np.array([0.2, -0.1, 0.35]) * 2 * np.pi / cl.lengths
        ctx.set_kpoint(k)
    f_ref, e_ref = O.nonlocal_force(psi, occ, _tab(t), st, cl.shape, st["dV"], occfac=2.0, wk=wk, kpt=k,
                                    lengths=cl.lengths)
    f, e = solver.NonlocalProjector(ctx).force(psi, occ, occfac=2.0, kpt=kpt, wk=wk)
    f_cref = ref.RefLynx(cl, pos, synth_psp8).nonlocal_force(psi, occ, kpt=k, wk=wk)
    assert f.shape == f_cref.shape
    assert np.abs(f - f_cref).max() <= 1e-10 * np.abs(f_cref).max()
    assert np.abs(f - f_ref).max() <= 1e-10 * np.abs(f_ref).max()
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
