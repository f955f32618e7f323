"""CPU tests of the C ABI library and the host-side set-up (no GPU needed).

* liblynxb200.so loads and exports every entry point include/lynx_b200.h declares;
* lynx_create / lynx_grid_info / lynx_stencil_coeffs (host-only) match the reference;
* lynx_fermi_level / lynx_occupations match the reference's Occupation;
* argument errors come back as status codes with a message;
* the projector tables and k-points built by lynx_b200 match the reference's.
"""
import ctypes
import os
import re

import numpy as np
import pytest

from lynx_b200 import _lib
from lynx_b200 import cell as C
from lynx_b200 import pseudo as P

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def golden(name):
    return dict(np.load(os.path.join(HERE, "golden", name)))


def header_symbols():
    with open(os.path.join(ROOT, "include", "lynx_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"LYNX_API\s+[\w\s\*]*?\b(lynx_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.EXPORTED)


def _ctx(g, orthogonal):
    lib = _lib.load()
    h = ctypes.c_void_p()
    lat = np.ascontiguousarray(g["latvec"], dtype=np.float64)
    nx, ny, nz = (int(v) for v in g["shape"])
    _lib.check(lib.lynx_create(ctypes.byref(h), 0, nx, ny, nz, 12, _lib.dptr(lat), int(orthogonal), None))
    return lib, h


@pytest.mark.parametrize("case,orth", [("golden_si8.npz", True), ("golden_fcc.npz", False)])
def test_create_grid_and_stencil(case, orth):
    g = golden(case)
    lib, h = _ctx(g, orth)
    try:
        nd, dV, me = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        _lib.check(lib.lynx_grid_info(h, ctypes.byref(nd), ctypes.byref(dV), ctypes.byref(me)))
        assert nd.value == int(np.prod(g["shape"]))
        assert abs(dV.value - float(g["dV"])) < 1e-15
        assert abs(me.value - float(g["st_max_eigval"])) < 1e-11
        out = {k: np.zeros(7) for k in ("D2x", "D2y", "D2z", "D2xy", "D2xz", "D2yz", "D1x", "D1y", "D1z")}
        _lib.check(lib.lynx_stencil_coeffs(h, *[_lib.dptr(out[k]) for k in
                                                ("D2x", "D2y", "D2z", "D2xy", "D2xz", "D2yz", "D1x", "D1y", "D1z")]))
        for k, v in out.items():
            np.testing.assert_allclose(v, g["st_" + k], rtol=1e-13, atol=1e-13)
    finally:
        lib.lynx_destroy(h)


def test_bad_arguments_return_status():
    lib = _lib.load()
    h = ctypes.c_void_p()
    lat = np.eye(3) * 10.0
    rc = lib.lynx_create(ctypes.byref(h), 0, 20, 20, 20, 11, _lib.dptr(lat), 1, None)
    assert rc == _lib.LYNX_ERR_BAD_ARG
    assert b"FD order" in lib.lynx_last_error()
    rc = lib.lynx_create(ctypes.byref(h), 0, 0, 20, 20, 12, _lib.dptr(lat), 1, None)
    assert rc == _lib.LYNX_ERR_BAD_ARG
    coplanar = np.array([[1.0, 0, 0], [0, 1.0, 0], [1.0, 1.0, 0]])
    rc = lib.lynx_create(ctypes.byref(h), 0, 20, 20, 20, 12, _lib.dptr(coplanar), 0, None)
    assert rc == _lib.LYNX_ERR_BAD_ARG
    assert lib.lynx_status_string(_lib.LYNX_ERR_CHOL_FAIL) == b"Cholesky factorization failed"


def test_fermi_level_and_occupations_match_reference():
    from lynx_b200 import solver
    g = golden("golden_occupation.npz")
    for ci in range(4):
        ne, beta, fd = g[f"occ{ci}_args"]
        e, w = g[f"occ{ci}_eig"], g[f"occ{ci}_w"]
        sm = "fermi-dirac" if fd else "gaussian"
        ef = solver.fermi_level(e, w, ne, beta, sm)
        f = solver.occupations(e, ef, beta, sm)
        assert abs(float(np.sum(w * f)) - ne) < 1e-10
        np.testing.assert_allclose(f, g[f"occ{ci}_f"], atol=1e-12)
        if ci != 0:  # case 0 has a gap >> 1/beta: every point of the gap is a root
            assert abs(ef - float(g[f"occ{ci}_ef"][0])) < 1e-11


def test_fermi_level_errors():
    from lynx_b200 import solver
    with pytest.raises(_lib.LynxError) as e:
        solver.fermi_level([0.0, 1.0], [2.0, 2.0], 10.0, 100.0)  # more electrons than states hold
    assert e.value.status == _lib.LYNX_ERR_BRACKET


@pytest.mark.parametrize("case", ["golden_si8.npz", "golden_fcc.npz"])
def test_projector_tables_match_reference(case, synth_psp8):
    g = golden(case)
    orth = case == "golden_si8.npz"
    cl = C.Cell(g["latvec"], tuple(int(v) for v in g["shape"]), orth, (0, 0, 0), 12)
    tab = P.nonlocal_tables(cl, g["positions"], P.read_psp8(synth_psp8))
    np.testing.assert_array_equal(tab.img_atom, g["nl_img_atom"])
    np.testing.assert_array_equal(tab.img_ndc, g["nl_img_ndc"])
    np.testing.assert_array_equal(tab.gpos, g["nl_gpos"])
    np.testing.assert_allclose(tab.img_shift, g["nl_img_shift"], atol=1e-12)
    np.testing.assert_allclose(tab.chi, g["nl_chi"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(tab.gamma, g["nl_gamma"], rtol=1e-15)


def test_kpoints_match_reference():
    g = golden("golden_si8.npz")
    cl = C.Cell(g["latvec"], tuple(int(v) for v in g["shape"]))
    for tag, grid, shift in (("kp444", (4, 4, 4), (0, 0, 0)), ("kp444s", (4, 4, 4), (0.5, 0.5, 0.5)),
                             ("kp321", (3, 2, 1), (0, 0, 0))):
        kc, kr, w = C.kpoints_mp(cl, grid, shift)
        np.testing.assert_allclose(kc, g[tag + "_cart"], atol=1e-14)
        np.testing.assert_array_equal(w, g[tag + "_w"])
    f = golden("golden_fcc.npz")
    clf = C.Cell(f["latvec"], tuple(int(v) for v in f["shape"]), False)
    kc, _, w = C.kpoints_mp(clf, (4, 4, 4))
    assert len(w) == 36 and abs(w.sum() - 64) < 1e-12
    np.testing.assert_allclose(kc, f["kp444_cart"], atol=1e-14)


def test_psp8_reader(synth_psp8):
    psp = P.read_psp8(synth_psp8)
    assert psp.lmax == 2 and psp.lloc == 4 and psp.ppl == [2, 2, 2]
    assert psp.nproj_per_atom == 18
    assert abs(psp.rc_max - 1.99) < 1e-12  # last grid point with |p_l| > 1e-12
    assert psp.udv[0][0][0] == psp.udv[0][0][1]  # r = 0 value copied from r = dr


def test_spline_reproduces_cubics():
    # a not-a-knot cubic spline is exact for cubic polynomials
    x = np.linspace(0.0, 3.0, 31)
    y = 1.0 - 2.0 * x + 0.5 * x ** 2 - 0.3 * x ** 3
    s = P.spline_slopes(x, y)
    xi = np.linspace(0.05, 2.95, 97)
    np.testing.assert_allclose(P.spline_eval(x, y, s, xi), 1.0 - 2.0 * xi + 0.5 * xi ** 2 - 0.3 * xi ** 3,
                               atol=1e-12)
