"""ctypes binding of liblynxb200.so (the C ABI declared in include/lynx_b200.h).

The shared library is built in-tree (``make -C lynx_b200/csrc``).  Loading fails
loudly when it is missing: there is no CPU fallback for any operator.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblynxb200.so")

LYNX_OK = 0
LYNX_ERR_BAD_ARG = 1
OPT_AUTOTUNE = 1
OPT_FUSE_NONLOCAL = 2
OPT_TC_RAYLEIGH_RITZ = 3
OPT_COMPACT_GATHER = 4
OPT_POISSON_DIRECT = 5
OPT_STENCIL_SHAPE = 6
OPT_HOST_COPY_BLOCK = 7
LYNX_ERR_CUDA = 2
LYNX_ERR_OOM = 3
LYNX_ERR_CHOL_FAIL = 4
LYNX_ERR_EIG_FAIL = 5
LYNX_ERR_NONFINITE = 6
LYNX_ERR_TIMEOUT = 7
LYNX_ERR_NOT_SETUP = 8
LYNX_ERR_UNSUPPORTED = 9
LYNX_ERR_BRACKET = 10

PREC_FP64 = 0
PREC_MIXED = 1
BC_PERIODIC = 0
BC_DIRICHLET = 1
SMEAR_GAUSSIAN = 0
SMEAR_FERMI_DIRAC = 1


class LynxError(RuntimeError):
    """A lynx_b200 entry point returned a non-OK status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"lynx_b200 status {status}: {message}")
        self.status = status


_c_int = ctypes.c_int
_c_double = ctypes.c_double
_p = ctypes.c_void_p
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes)
_SIGNATURES = {
    "lynx_status_string": (ctypes.c_char_p, [_c_int]),
    "lynx_last_error": (ctypes.c_char_p, []),
    "lynx_version": (_c_int, []),
    "lynx_create": (_c_int, [ctypes.POINTER(_p), _c_int, _c_int, _c_int, _c_int, _c_int, _pd, _c_int, _pi]),
    "lynx_destroy": (_c_int, [_p]),
    "lynx_set_stream": (_c_int, [_p, _p]),
    "lynx_grid_info": (_c_int, [_p, _pi, _pd, _pd]),
    "lynx_stencil_coeffs": (_c_int, [_p, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    "lynx_set_nonlocal": (_c_int, [_p, _c_int, _pi, _pi, _pd, _pi, _pd, _c_int, _pi, _pd]),
    "lynx_set_kpoint": (_c_int, [_p, _pd]),
    "lynx_hamiltonian_apply": (_c_int, [_p, _p, _p, _p, _c_int, _c_int, _c_double]),
    "lynx_hamiltonian_apply_kpt": (_c_int, [_p, _p, _p, _p, _c_int, _c_int, _c_double]),
    "lynx_nonlocal_apply": (_c_int, [_p, _p, _p, _c_int, _c_int]),
    "lynx_nonlocal_apply_noalloc": (_c_int, [_p, _p, _p, _c_int, _c_int]),
    "lynx_set_option": (_c_int, [_p, _c_int, _c_int]),
    "lynx_eigensolver_solve_batch": (_c_int, [_p, _c_int, _p, _p, _p, _p, _p, _p, _p, _p, _p, _c_int, _c_int, _p]),
    "lynx_nonlocal_force": (_c_int, [_p, _p, _c_int, _c_int, _p, ctypes.c_double, _p, _p]),
    "lynx_nonlocal_force_kpt": (_c_int, [_p, _p, _c_int, _c_int, _p, ctypes.c_double, _p, _p]),
    "lynx_kinetic_nonlocal_stress": (_c_int, [_p, _p, _c_int, _c_int, _p, ctypes.c_double, _p, _p, _p]),
    "lynx_randomize_orbitals": (_c_int, [_p, _p, _c_int, _c_int, ctypes.c_ulonglong, _c_int]),
    "lynx_randomize_orbitals_all": (_c_int, [_p, _p, _c_int, _c_int, _c_int, _c_int, _c_int]),
    "lynx_kinetic_nonlocal_stress_kpt": (_c_int, [_p, _p, _c_int, _c_int, _p, ctypes.c_double, _p, _p, _p]),
    "lynx_nonlocal_apply_kpt": (_c_int, [_p, _p, _p, _c_int, _c_int]),
    "lynx_chebyshev_filter": (_c_int, [_p, _p, _p, _p, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _c_int]),
    "lynx_chebyshev_filter_kpt": (_c_int, [_p, _p, _p, _p, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _c_int]),
    "lynx_eigensolver_solve": (_c_int, [_p, _p, _pd, _p, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _c_int, _pd]),
    "lynx_eigensolver_solve_kpt": (_c_int, [_p, _p, _pd, _p, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _c_int, _pd]),
    "lynx_eigensolver_solve_host": (_c_int, [_p, _pd, _pd, _pd, _c_int, _c_int, _c_double, _c_double, _c_double, _c_int, _c_int, _pd]),
    "lynx_lanczos_bounds": (_c_int, [_p, _p, _c_double, _c_int, _pd, _pd]),
    "lynx_lanczos_bounds_kpt": (_c_int, [_p, _p, _c_double, _c_int, _pd, _pd]),
    "lynx_fermi_level": (_c_int, [_pd, _pd, _c_int, _c_double, _c_double, _c_int, _pd]),
    "lynx_occupations": (_c_int, [_pd, _c_int, _c_double, _c_double, _c_int, _pd]),
    "lynx_time_filter_step": (_c_int, [_p, _p, _c_int, _c_int, _c_int, _c_int, _pd]),
    "lynx_launch_count": (ctypes.c_longlong, [_c_int]),
    "lynx_gram_mixed": (_c_int, [_p, _p, _p, ctypes.c_longlong, ctypes.c_longlong, _c_int, _c_double, _p, _p]),
    "lynx_rotate_mixed": (_c_int, [_p, _p, ctypes.c_longlong, ctypes.c_longlong, _p, _p, _c_int, _p,
                                   ctypes.c_longlong]),
    "lynx_selftest_wait_timeout": (_c_int, [_p, _c_int]),
    "lynx_electron_density": (_c_int, [_p, _p, _c_int, _c_int, _pd, _c_double, _p, _c_int, _c_int]),
    "lynx_eigensolver_solve_density": (_c_int, [_p, _p, _pd, _p, _c_int, _c_int, _c_double, _c_double, _c_double,
                                                _c_int, _c_int, _pd, _c_double, _c_double, _c_int, _c_double, _p,
                                                _pd]),
    "lynx_xc_gga_pbe": (_c_int, [_p, _p, _p, _p, _p, _p]),
    "lynx_poisson_solve": (_c_int, [_p, _p, _p, _c_double, _c_int, _pi]),
    "lynx_effective_potential": (_c_int, [_p, _p, _p, _p, _c_double, _p, _p, _p, _p, _pi]),
}

EXPORTED = tuple(_SIGNATURES)

_lib = None


def load() -> ctypes.CDLL:
    """Load liblynxb200.so (once) and declare the ABI.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `make -C lynx_b200/csrc` "
            "(lynx_b200 has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != LYNX_OK:
        lib = load()
        raise LynxError(status, lib.lynx_last_error().decode())


def dptr(arr) -> ctypes.POINTER(ctypes.c_double):
    """Pointer to a C-contiguous float64 numpy array."""
    return arr.ctypes.data_as(_pd)


def iptr(arr) -> ctypes.POINTER(ctypes.c_int):
    return arr.ctypes.data_as(_pi)
