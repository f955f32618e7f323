"""Pin the numpy oracle (oracle/chefsi_oracle.py) to the reference's golden vectors.

The golden vectors in tests/golden/*.npz were produced by the reference LYNX CPU
sources themselves (tests/golden/make_golden.py).  CPU only.
"""
import os

import numpy as np
import pytest

from oracle import chefsi_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name)))


@pytest.fixture(scope="module")
def si8():
    return load("golden_si8.npz")


@pytest.fixture(scope="module")
def fcc():
    return load("golden_fcc.npz")


def tables(g):
    return {k[3:]: g[k] for k in g if k.startswith("nl_")}


def op(g, orthogonal=True):
    return O.Operator(g["latvec"], tuple(g["shape"]), int(g["fd_order"]), orthogonal, tables(g))


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(b).max())


def test_fd_weights_order6_closed_form():
    # tests/unit/test_FDStencil.cpp: order-6 weights
    w1, w2 = O.fd_weights(6)
    np.testing.assert_allclose(w1[1:], [0.75, -0.15, 1.0 / 60.0], rtol=1e-13)
    np.testing.assert_allclose(w2, [-(2 + 0.5 + 2.0 / 9.0), 1.5, -0.15, 0.1 / 9.0], rtol=1e-13)
    assert abs(w2[0] + 2 * w2[1:].sum()) < 1e-13


def test_fd_weights_order12_closed_form():
    # central-difference weights, w2[p] = 2 (-1)^(p+1) (n!)^2 / (p^2 (n-p)! (n+p)!), n = 6
    from fractions import Fraction
    from math import factorial as F
    n = 6
    exp = [Fraction(0)] * (n + 1)
    for p in range(1, n + 1):
        exp[p] = Fraction(2 * (-1) ** (p + 1) * F(n) ** 2, p * p * F(n - p) * F(n + p))
        exp[0] -= Fraction(2, p * p)
    _, w2 = O.fd_weights(12)
    np.testing.assert_allclose(w2, [float(v) for v in exp], rtol=1e-14)


@pytest.mark.parametrize("case,orth", [("si8", True), ("fcc", False)])
def test_stencil(case, orth, si8, fcc):
    g = si8 if case == "si8" else fcc
    st = O.stencil(g["latvec"], tuple(g["shape"]), 12, orth)
    for k in ("D2x", "D2y", "D2z", "D1x", "D1y", "D1z", "D2xy", "D2xz", "D2yz", "w1", "w2"):
        np.testing.assert_allclose(st[k], g["st_" + k], rtol=1e-13, atol=1e-13)
    assert abs(st["max_eigval"] - float(g["st_max_eigval"])) < 1e-11
    assert abs(st["dV"] - float(g["dV"])) < 1e-15


def test_hamiltonian_real(si8):
    H = op(si8)
    y = H.apply(si8["psi"], si8["veff"], 0.25)
    assert rel(y, si8["hpsi"]) < 1e-13


def test_hamiltonian_kpt(si8):
    H = op(si8)
    y = H.apply(si8["psiz"], si8["veff"], 0.1, kpt=si8["kpt"])
    assert rel(y, si8["hpsiz"]) < 1e-13


def test_nonlocal(si8):
    H = op(si8)
    y = O.nonlocal_apply(si8["psi"], np.zeros_like(si8["psi"]), tables(si8), H.dV)
    assert rel(y, si8["vnlpsi"]) < 1e-13


def test_hamiltonian_nonorthogonal(fcc):
    H = op(fcc, orthogonal=False)
    assert rel(H.apply(fcc["psi"], fcc["veff"]), fcc["hpsi"]) < 1e-12
    assert rel(H.apply(fcc["psiz"], fcc["veff"], kpt=fcc["kpt"]), fcc["hpsiz"]) < 1e-12


def test_chebyshev_filter(si8):
    H = op(si8)
    lc, lo, hi, m = si8["filter_args"]
    Y = O.chebyshev_filter(H, si8["psi"], si8["veff"], lc, lo, hi, int(m))
    assert rel(Y, si8["filter_y"]) < 1e-11
    lc, lo, hi, m = si8["filterz_args"]
    Yz = O.chebyshev_filter(H, si8["psiz"], si8["veff"], lc, lo, hi, int(m), kpt=si8["kpt"])
    assert rel(Yz, si8["filterz_y"]) < 1e-11


def test_solve(si8):
    H = op(si8)
    lc, lo, hi, m = si8["solve_args"]
    psi, eig, lc_next = O.solve(H, si8["solve_psi0"], si8["veff"], lc, lo, hi, int(m))
    np.testing.assert_allclose(eig, si8["solve_eig"], atol=1e-10)
    assert abs(lc_next - float(si8["solve_lc"][0])) < 1e-10
    # Ritz vectors agree up to sign (non-degenerate Ritz values)
    ref = si8["solve_psi"]
    for j in range(ref.shape[1]):
        s = np.sign(np.dot(psi[:, j], ref[:, j]))
        assert rel(s * psi[:, j], ref[:, j]) < 1e-7


def test_lanczos(si8):
    H = op(si8)
    lo, hi = O.lanczos_bounds(H, si8["veff"])
    np.testing.assert_allclose([lo, hi], si8["lanczos"], rtol=1e-9)
    loz, hiz = O.lanczos_bounds(H, si8["veff"], kpt=si8["kpt"])
    np.testing.assert_allclose([loz, hiz], si8["lanczos_kpt"], rtol=1e-9)


@pytest.mark.parametrize("tag,shift", [("kp444", (0, 0, 0)), ("kp444s", (0.5, 0.5, 0.5)), ("kp321", (0, 0, 0))])
def test_kpoints(si8, tag, shift):
    grid = {"kp444": (4, 4, 4), "kp444s": (4, 4, 4), "kp321": (3, 2, 1)}[tag]
    L = np.linalg.norm(si8["latvec"], axis=1)
    kc, kr, w = O.kpoints(L, grid, shift)
    np.testing.assert_allclose(kc, si8[tag + "_cart"], atol=1e-14)
    np.testing.assert_allclose(kr, si8[tag + "_red"], atol=1e-14)
    np.testing.assert_array_equal(w, si8[tag + "_w"])


def test_kpoints_fcc(fcc):
    L = np.linalg.norm(fcc["latvec"], axis=1)
    kc, kr, w = O.kpoints(L, (4, 4, 4))
    np.testing.assert_allclose(kc, fcc["kp444_cart"], atol=1e-14)
    np.testing.assert_array_equal(w, fcc["kp444_w"])
    assert len(w) == 36  # 64 points, time-reversal reduced


def test_fermi_level():
    g = load("golden_occupation.npz")
    for ci in range(4):
        ne, beta, fd = g[f"occ{ci}_args"]
        e, w = g[f"occ{ci}_eig"], g[f"occ{ci}_w"]
        ef = O.fermi_level(e, w, ne, beta, bool(fd))
        f = O.smearing(e - ef, beta, bool(fd))
        # Ef itself is only determined where N(Ef) is not flat: in a gap much wider than
        # 1/beta any point of the gap is a root, so the occupations are what must agree.
        assert abs(float(np.sum(w * f)) - ne) < 1e-10
        np.testing.assert_allclose(f, g[f"occ{ci}_f"], atol=1e-12)
        np.testing.assert_allclose(O.smearing(e - g[f"occ{ci}_ef"][0], beta, bool(fd)), g[f"occ{ci}_f"],
                                   atol=1e-14)
        if ci != 0:
            assert abs(ef - float(g[f"occ{ci}_ef"][0])) < 1e-11
