"""Python mirror of the B200 Simint engine's C API.

The product is libsimint_b200.so (C ABI, include/simint/*.h and
include/simint_b200.h).  This module binds it with ctypes so the tests and
bench.py call exactly what a C host would call:

    lib = simint_b200.load()
    lib.simint_init()
    ... simint_create_multi_shellpair(...), simint_compute_eri(...)

There is no CPU fallback: if the library or a CUDA device is missing the
calls fail (negative return codes, simint_b200_last_error()).
"""

import ctypes as C
import os

import numpy as np

from .capi import (SimintShell, SimintMultiShellpair, ShellSet, ShellP, PairP,
                   declare_shell_api, pair_arrays, padded_nprim,
                   SIMINT_SCREEN_NONE, SIMINT_SCREEN_SCHWARZ, SIMINT_SCREEN_FASTSCHWARZ)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(os.path.dirname(HERE), "libsimint_b200.so")

PSI4, GAMESS = 0, 1
FP64, MIXED = 0, 1

_lib = None
_dp = C.POINTER(C.c_double)

EXPORTED = None  # filled from the headers by tests


def load(path=LIBPATH):
    """Load libsimint_b200.so (raises OSError when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("libsimint_b200.so not built: run simint-generator_b200/build.py")
    lib = C.CDLL(path)
    declare_shell_api(lib)
    lib.simint_init.restype = None
    lib.simint_finalize.restype = None
    lib.simint_compute_eri.argtypes = [PairP, PairP, C.c_double, _dp, _dp]
    lib.simint_compute_eri.restype = C.c_int
    lib.simint_compute_eri_deriv.argtypes = [C.c_int, PairP, PairP, C.c_double, _dp, _dp]
    lib.simint_compute_eri_deriv.restype = C.c_int
    lib.simint_eri_worksize.argtypes = [C.c_int, C.c_int]
    lib.simint_eri_worksize.restype = C.c_size_t
    lib.simint_eri_workmem.argtypes = [C.c_int, C.c_int]
    lib.simint_eri_workmem.restype = C.c_size_t
    lib.simint_b200_set_ordering.argtypes = [C.c_int]
    lib.simint_b200_set_ordering.restype = C.c_int
    lib.simint_b200_get_ordering.restype = C.c_int
    lib.simint_b200_set_precision.argtypes = [C.c_int, C.c_double]
    lib.simint_b200_set_precision.restype = C.c_int
    lib.simint_b200_get_precision.restype = C.c_int
    lib.simint_b200_last_error.restype = C.c_char_p
    lib.simint_b200_launch_count.restype = C.c_longlong
    _lib = lib
    return lib


def last_error():
    return load().simint_b200_last_error().decode()


def ncart(l):
    return (l + 1) * (l + 2) // 2


def make_pairs(lib, shells, pairs, screen=SIMINT_SCREEN_NONE):
    """simint_create_multi_shellpair2 over an explicit list of (i, j)."""
    P = SimintMultiShellpair()
    lib.simint_initialize_multi_shellpair(C.byref(P))
    arr = shells.pair_list(pairs)
    lib.simint_create_multi_shellpair2(len(pairs), C.cast(arr, ShellP), C.byref(P), screen)
    return P


def compute_eri(P, Q, screen_tol=0.0, deriv=0, lib=None):
    """simint_compute_eri(_deriv) into a fresh numpy array.

    Returns (ret, out).  ret < 0 other than -1 raises RuntimeError."""
    lib = lib or load()
    n = P.nshell12_clip * Q.nshell12_clip * ncart(P.am1) * ncart(P.am2) * ncart(Q.am1) * ncart(Q.am2)
    out = np.zeros(n * (12 if deriv else 1))
    r = lib.simint_compute_eri_deriv(deriv, C.byref(P), C.byref(Q), screen_tol, None,
                                     out.ctypes.data_as(_dp))
    if r < -1:
        raise RuntimeError("simint_compute_eri_deriv failed (%d): %s" % (r, last_error()))
    return r, out
