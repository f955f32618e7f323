"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs oracle/_ref/libref_lynx.so (the reference LYNX CPU sources compiled unmodified by
oracle/Makefile) on small seeded inputs and stores inputs and outputs as .npz files.
Re-run after rebuilding the oracle:  python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lynx_b200 import cell as C  # noqa: E402
from lynx_b200 import pseudo as P  # noqa: E402
from oracle import ref  # noqa: E402


def tables(R):
    t = R.nl_tables()
    return {"nl_" + k: v for k, v in t.items()}


def make_si8(psp):
    cl, pos = C.diamond_si(1, 14, displace=0.05, seed=3)
    cl.shape = (14, 15, 16)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=3)
    R = ref.RefLynx(cl, pos, psp)
    st = R.stencil()
    out = dict(latvec=cl.latvec, shape=np.array(cl.shape), fd_order=12, positions=pos, veff=V, dV=R.dV)
    out.update({"st_" + k: v for k, v in st.items()})
    out.update(tables(R))
    psi = C.random_orbitals(R.nd, 4, seed=11)
    psiz = C.random_orbitals(R.nd, 2, seed=12, complex_=True)
    k = np.array([0.11, -0.23, 0.31]) * 2 * np.pi / cl.lengths
    out.update(psi=psi, psiz=psiz, kpt=k)
    out["hpsi"] = R.h_apply(psi, V, 0.25)
    out["hpsiz"] = R.h_apply_kpt(psiz, V, k, 0.1)
    out["vnlpsi"] = R.nl_apply(psi, np.zeros_like(psi))
    lo, hi = R.lanczos(V)
    out["lanczos"] = np.array([lo, hi])
    loz, hiz = R.lanczos(V, kpt=k)
    out["lanczos_kpt"] = np.array([loz, hiz])
    lc = 0.5 * (lo + hi)
    out["filter_args"] = np.array([lc, lo, hi, 6])
    out["filter_y"] = R.chebyshev_filter(psi, V, lc, lo, hi, 6)
    lcz = 0.5 * (loz + hiz)
    out["filterz_args"] = np.array([lcz, loz, hiz, 4])
    out["filterz_y"] = R.chebyshev_filter_kpt(psiz, V, lcz, loz, hiz, 4, k)
    psi6 = C.random_orbitals(R.nd, 6, seed=13)
    out["solve_psi0"] = psi6
    out["solve_args"] = np.array([lc, lo, hi, 8])
    p6, e6 = R.solve(psi6, V, lc, lo, hi, 8)
    out["solve_psi"] = p6
    out["solve_eig"] = e6
    out["solve_lc"] = np.array([ref.lib().ref_lambda_cutoff()])
    kc, kr, w = R.kpoints((4, 4, 4))
    out.update(kp444_cart=kc, kp444_red=kr, kp444_w=w)
    kc, kr, w = R.kpoints((4, 4, 4), (0.5, 0.5, 0.5))
    out.update(kp444s_cart=kc, kp444s_red=kr, kp444s_w=w)
    kc, kr, w = R.kpoints((3, 2, 1))
    out.update(kp321_cart=kc, kp321_red=kr, kp321_w=w)
    return out


def make_fcc(psp):
    cl, pos = C.fcc_si_primitive(14)
    V = C.synthetic_veff(cl, pos, noise=1e-3, seed=4)
    R = ref.RefLynx(cl, pos, psp)
    st = R.stencil()
    out = dict(latvec=cl.latvec, shape=np.array(cl.shape), fd_order=12, positions=pos, veff=V, dV=R.dV)
    out.update({"st_" + k: v for k, v in st.items()})
    out.update(tables(R))
    psi = C.random_orbitals(R.nd, 2, seed=21)
    psiz = C.random_orbitals(R.nd, 2, seed=22, complex_=True)
    k = np.array([0.25, 0.0, -0.25]) * 2 * np.pi / cl.lengths
    out.update(psi=psi, psiz=psiz, kpt=k)
    out["hpsi"] = R.h_apply(psi, V, 0.0)
    out["hpsiz"] = R.h_apply_kpt(psiz, V, k, 0.0)
    kc, kr, w = R.kpoints((4, 4, 4))
    out.update(kp444_cart=kc, kp444_red=kr, kp444_w=w)
    return out


def make_occupation():
    rng = np.random.default_rng(5)
    out = {}
    cases = []
    for ci, (n, beta, fd) in enumerate([(24, 1000.0, 1), (160, 315.77, 1), (40, 50.0, 0), (16 * 36, 1000.0, 1)]):
        e = np.sort(rng.uniform(-0.4, 0.6, n))
        w = np.full(n, 2.0) if ci != 3 else np.repeat(rng.choice([1.0, 2.0], 36) / 64.0 * 2.0, 16)
        ne = float(np.sum(w[: n // 2]))
        ef = ref.fermi_level(e, w, ne, beta, bool(fd))
        out[f"occ{ci}_eig"] = e
        out[f"occ{ci}_w"] = w
        out[f"occ{ci}_args"] = np.array([ne, beta, fd])
        out[f"occ{ci}_ef"] = np.array([ef])
        out[f"occ{ci}_f"] = np.array([ref.smearing(x - ef, beta, bool(fd)) for x in e])
    return out


def main():
    with tempfile.TemporaryDirectory() as td:
        psp = P.synthetic_si_psp8(os.path.join(td, "Si_synthetic.psp8"))
        np.savez_compressed(os.path.join(HERE, "golden_si8.npz"), **make_si8(psp))
        np.savez_compressed(os.path.join(HERE, "golden_fcc.npz"), **make_fcc(psp))
        np.savez_compressed(os.path.join(HERE, "golden_occupation.npz"), **make_occupation())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
