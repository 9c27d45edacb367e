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
_libs = {}
_dp = C.POINTER(C.c_double)

EXPORTED = None  # filled from the headers by tests


def load(path=LIBPATH):
    """Load libsimint_b200.so (raises OSError when it is not built); one
    handle per path."""
    global _lib
    if path == LIBPATH and _lib is not None:
        return _lib
    if path in _libs:
        return _libs[path]
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
    if path == LIBPATH:
        _lib = lib
    _libs[path] = lib
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


OEI_OVERLAP, OEI_KINETIC, OEI_POTENTIAL = 0, 1, 2


def _centres(centres):
    """(x, y, z, Z) rows -> four contiguous arrays (kept alive by the caller)."""
    c = np.ascontiguousarray(np.asarray(centres, float).reshape(-1, 4).T)
    return c, [c[k].ctypes.data_as(_dp) for k in (3, 0, 1, 2)]


def compute_oei(kind, S, a, b, centres=None, lib=None):
    """simint_compute_overlap / _ke / _potential for shells a, b of S (the
    reference's per-pair interface); returns (ret, block)."""
    lib = lib or load()
    n = ncart(S.arr[a].am) * ncart(S.arr[b].am)
    out = np.zeros(n)
    if kind == OEI_OVERLAP:
        lib.simint_compute_overlap.argtypes = [ShellP, ShellP, _dp]
        r = lib.simint_compute_overlap(S.ptr(a), S.ptr(b), out.ctypes.data_as(_dp))
    elif kind == OEI_KINETIC:
        lib.simint_compute_ke.argtypes = [ShellP, ShellP, _dp]
        r = lib.simint_compute_ke(S.ptr(a), S.ptr(b), out.ctypes.data_as(_dp))
    else:
        keep, (Z, x, y, z) = _centres(centres if centres is not None else np.zeros((0, 4)))
        lib.simint_compute_potential.argtypes = [C.c_int, _dp, _dp, _dp, _dp, ShellP, ShellP, _dp]
        r = lib.simint_compute_potential(keep.shape[1], Z, x, y, z, S.ptr(a), S.ptr(b),
                                         out.ctypes.data_as(_dp))
    return r, out


def oei_matrix(kind, S, centres, dev_out, stream=0, lib=None):
    """simint_b200_oei_matrix: the nbf x nbf matrix of every shell of S into
    device memory at dev_out; returns the launch count."""
    lib = lib or load()
    keep, (Z, x, y, z) = _centres(centres if centres is not None else np.zeros((0, 4)))
    lib.simint_b200_oei_matrix.argtypes = [C.c_int, C.c_int, ShellP, C.c_int, _dp, _dp, _dp, _dp,
                                           C.c_void_p, C.c_void_p]
    r = lib.simint_b200_oei_matrix(kind, S.n, S.ptr(0), keep.shape[1], Z, x, y, z,
                                   C.c_void_p(dev_out), C.c_void_p(stream))
    if r < 0:
        raise RuntimeError("simint_b200_oei_matrix failed: " + last_error())
    return r


def count_primq(P, Q, screen_tol, lib=None):
    lib = lib or load()
    lib.simint_b200_count_primq.argtypes = [PairP, PairP, C.c_double]
    lib.simint_b200_count_primq.restype = C.c_longlong
    return lib.simint_b200_count_primq(C.byref(P), C.byref(Q), screen_tol)


def fma_peak(fp32=False, lib=None):
    lib = lib or load()
    lib.simint_b200_fma_peak.argtypes = [C.c_int]
    lib.simint_b200_fma_peak.restype = C.c_double
    return lib.simint_b200_fma_peak(1 if fp32 else 0)


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


VAR_DEFAULT, VAR_STRAIGHT, VAR_COOP1, VAR_GENERIC, VAR_STRAIGHT64 = 0, 1, 3, 4, 5
VAR_WARP, VAR_WARP64 = 6, 7                 # register kernel, one warp per shell quartet
VAR_COOP2 = {1: 21, 2: 22, 4: 24, 8: 28}          # cooperative kernel, 256 threads, batch B
VAR_COOP2_128 = {1: 41, 2: 42, 4: 44, 8: 48}      # cooperative kernel, 128 threads, batch B
VAR_COOP2_64 = {1: 61, 2: 62, 4: 64, 8: 68}       # cooperative kernel, 64 threads, batch B
VAR_COL = {4: 81, 8: 82}                          # column kernel, NP primitive quartets per batch
VAR_COL_GROUPS = 83                               # column kernel, 4 per batch, two thread groups per CTA


PAIR_FILL_AUTO, PAIR_FILL_HOST, PAIR_FILL_GPU = 0, 1, 2


def set_pair_fill(mode, lib=None):
    """Where simint_create_multi_shellpair(2) computes the Gaussian-product
    fill (simint_b200_set_pair_fill): PAIR_FILL_AUTO, _HOST or _GPU; returns
    the C status."""
    lib = lib or load()
    lib.simint_b200_set_pair_fill.argtypes = [C.c_int]
    lib.simint_b200_set_pair_fill.restype = C.c_int
    return lib.simint_b200_set_pair_fill(mode)


def get_pair_fill(lib=None):
    lib = lib or load()
    lib.simint_b200_get_pair_fill.restype = C.c_int
    return lib.simint_b200_get_pair_fill()


def get_variant(am, deriv=0, prec=0, lib=None):
    """Kernel variant in force for a requested class (simint_b200_variant)."""
    lib = lib or load()
    lib.simint_b200_variant.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int]
    return lib.simint_b200_variant((C.c_int * 4)(*am), deriv, prec)


def set_variant(am, variant, deriv=0, prec=0, lib=None):
    """Pin the kernel variant of a requested class; returns the C status
    (0, or SIMINT_B200_ERR_ARG when the variant does not exist for it)."""
    lib = lib or load()
    lib.simint_b200_set_variant.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int]
    return lib.simint_b200_set_variant((C.c_int * 4)(*am), deriv, prec, variant)


class Basis:
    """simint_b200_basis: a device-resident, Schwarz-screened sweep."""

    def __init__(self, shells, screen_tol, max_am=4, lib=None):
        self.lib = lib or load()
        L = self.lib
        L.simint_b200_basis_create.argtypes = [C.c_int, ShellP, C.c_double, C.c_int]
        L.simint_b200_basis_create.restype = C.c_void_p
        L.simint_b200_basis_free.argtypes = [C.c_void_p]
        L.simint_b200_basis_nquartets.argtypes = [C.c_void_p]
        L.simint_b200_basis_nquartets.restype = C.c_longlong
        L.simint_b200_basis_nprimquartets.argtypes = [C.c_void_p]
        L.simint_b200_basis_nprimquartets.restype = C.c_longlong
        L.simint_b200_basis_output_size.argtypes = [C.c_void_p]
        L.simint_b200_basis_output_size.restype = C.c_longlong
        L.simint_b200_basis_nclass.argtypes = [C.c_void_p]
        L.simint_b200_basis_class_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                                   C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                                   C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        L.simint_b200_basis_quartet.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.POINTER(C.c_int)]
        L.simint_b200_basis_compute.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong, C.c_void_p]
        L.simint_b200_basis_checksums.argtypes = [C.c_void_p, _dp]
        L.simint_b200_basis_class_times.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong,
                                                    C.c_void_p, C.POINTER(C.c_float)]
        self.shells = shells
        self.h = L.simint_b200_basis_create(shells.n, shells.ptr(0), screen_tol, max_am)
        if not self.h:
            raise RuntimeError("simint_b200_basis_create failed: " + last_error())

    def close(self):
        if self.h:
            self.lib.simint_b200_basis_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nquartets(self):
        return self.lib.simint_b200_basis_nquartets(self.h)

    @property
    def nprimquartets(self):
        return self.lib.simint_b200_basis_nprimquartets(self.h)

    @property
    def output_size(self):
        return self.lib.simint_b200_basis_output_size(self.h)

    def classes(self):
        out = []
        for k in range(self.lib.simint_b200_basis_nclass(self.h)):
            am = (C.c_int * 4)()
            nq, npq, off = C.c_longlong(), C.c_longlong(), C.c_longlong()
            nout = C.c_int()
            self.lib.simint_b200_basis_class_info(self.h, k, am, C.byref(nq), C.byref(npq),
                                                  C.byref(nout), C.byref(off))
            out.append(dict(am=tuple(am), nquart=nq.value, nprimq=npq.value,
                            nout=nout.value, offset=off.value))
        return out

    def subsample(self, max_quartets):
        L = self.lib
        L.simint_b200_basis_subsample.argtypes = [C.c_void_p, C.c_longlong]
        r = L.simint_b200_basis_subsample(self.h, max_quartets)
        if r != 0:
            raise RuntimeError("subsample failed: " + last_error())

    def subsample_stride(self, stride, offset=0):
        self.lib.simint_b200_basis_subsample_stride.argtypes = [C.c_void_p, C.c_int, C.c_int]
        r = self.lib.simint_b200_basis_subsample_stride(self.h, stride, offset)
        if r != 0:
            raise RuntimeError("subsample_stride failed: " + last_error())

    def rows(self, k):
        """(first task, number of tasks) of every bra-pair row of class k."""
        L = self.lib
        L.simint_b200_basis_nrows.argtypes = [C.c_void_p, C.c_int]
        L.simint_b200_basis_row.argtypes = [C.c_void_p, C.c_int, C.c_int,
                                            C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        out = []
        for r in range(L.simint_b200_basis_nrows(self.h, k)):
            f, n = C.c_longlong(), C.c_longlong()
            L.simint_b200_basis_row(self.h, k, r, C.byref(f), C.byref(n))
            out.append((f.value, n.value))
        return out

    def class_full(self, k):
        self.lib.simint_b200_basis_class_full.argtypes = [C.c_void_p, C.c_int]
        self.lib.simint_b200_basis_class_full.restype = C.c_longlong
        return self.lib.simint_b200_basis_class_full(self.h, k)

    def count_primq(self):
        self.lib.simint_b200_basis_count_primq.argtypes = [C.c_void_p]
        self.lib.simint_b200_basis_count_primq.restype = C.c_longlong
        return self.lib.simint_b200_basis_count_primq(self.h)

    def quartet(self, k, q):
        sh = (C.c_int * 4)()
        r = self.lib.simint_b200_basis_quartet(self.h, k, q, sh)
        if r != 0:
            raise IndexError((k, q))
        return tuple(sh)

    def class_quartets(self, k, nquart):
        """(nquart, 4) int array: the shells of every quartet of class k."""
        sh = np.zeros((max(nquart, 1), 4), dtype=np.int32)
        self.lib.simint_b200_basis_class_quartets.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        r = self.lib.simint_b200_basis_class_quartets(self.h, k, C.c_void_p(sh.ctypes.data))
        if r != 0:
            raise IndexError(k)
        return sh[:nquart]

    def class_kets(self, k):
        """(n, 2) int array: the ket pair list of class k in stored order."""
        self.lib.simint_b200_basis_class_kets.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        n = self.lib.simint_b200_basis_class_kets(self.h, k, None)
        if n < 0:
            raise IndexError(k)
        sh = np.zeros((max(n, 1), 2), dtype=np.int32)
        self.lib.simint_b200_basis_class_kets(self.h, k, C.c_void_p(sh.ctypes.data))
        return sh[:n]

    def compute(self, prec, dev_ptr, ndoubles, stream=0):
        r = self.lib.simint_b200_basis_compute(self.h, prec, C.c_void_p(dev_ptr), ndoubles,
                                               C.c_void_p(stream))
        if r < 0:
            raise RuntimeError("simint_b200_basis_compute failed (%d): %s" % (r, last_error()))
        return r

    def autotune(self, prec, dev_ptr, ndoubles, stream=0):
        L = self.lib
        L.simint_b200_basis_autotune.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong, C.c_void_p]
        r = L.simint_b200_basis_autotune(self.h, prec, C.c_void_p(dev_ptr), ndoubles, C.c_void_p(stream))
        if r != 0:
            raise RuntimeError("autotune failed: " + last_error())

    def variant(self, am, prec, deriv=0):
        self.lib.simint_b200_variant.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int]
        return self.lib.simint_b200_variant((C.c_int * 4)(*am), deriv, prec)

    def checksums(self):
        """(nclass, 2): sum and sum of absolute values per class of the last
        compute; raises when a work-queue wait of the sweep ran out."""
        n = self.lib.simint_b200_basis_nclass(self.h)
        s = np.zeros(2 * max(n, 1))
        r = self.lib.simint_b200_basis_checksums(self.h, s.ctypes.data_as(_dp))
        if r != 0:
            raise RuntimeError("simint_b200_basis_checksums failed (%d): %s" % (r, last_error()))
        return s[:2 * n].reshape(n, 2)

    def fp32_counts(self):
        """Primitive quartets of the last compute that ran their VRR in FP32,
        per class (int64 array)."""
        n = self.lib.simint_b200_basis_nclass(self.h)
        c = np.zeros(max(n, 1), dtype=np.int64)
        self.lib.simint_b200_basis_fp32_counts.argtypes = [C.c_void_p, C.c_void_p]
        r = self.lib.simint_b200_basis_fp32_counts(self.h, C.c_void_p(c.ctypes.data))
        if r != 0:
            raise RuntimeError("simint_b200_basis_fp32_counts failed: " + last_error())
        return c[:n]

    def queue_probe(self, k, published, closed, wait_ms, dev_ptr, ndoubles):
        """simint_b200_basis_queue_probe: class k with a queue of `published`
        tasks, closed or open; returns the C status (published, or
        SIMINT_B200_ERR_TIMEOUT when a wait ran out)."""
        L = self.lib
        L.simint_b200_basis_queue_probe.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_int,
                                                    C.c_void_p, C.c_longlong]
        return L.simint_b200_basis_queue_probe(self.h, k, published, int(closed), wait_ms,
                                               C.c_void_p(dev_ptr), ndoubles)

    @property
    def nbf(self):
        self.lib.simint_b200_basis_nbf.argtypes = [C.c_void_p]
        return self.lib.simint_b200_basis_nbf(self.h)

    def jk(self, dev_out, ndoubles, dev_D, dev_J, dev_K, stream=0):
        """Coulomb and exchange matrices of density D from a full-layout
        sweep output (simint_b200_basis_jk); device pointers."""
        L = self.lib
        L.simint_b200_basis_jk.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]
        r = L.simint_b200_basis_jk(self.h, C.c_void_p(dev_out), ndoubles, C.c_void_p(dev_D),
                                   C.c_void_p(dev_J), C.c_void_p(dev_K), C.c_void_p(stream))
        if r < 0:
            raise RuntimeError("simint_b200_basis_jk failed: " + last_error())
        return r

    def compute_jk(self, prec, dev_D, dev_J, dev_K, dev_scratch, scratch_doubles, stream=0):
        """The sweep and its J/K digestion chunk by chunk through a scratch
        buffer (simint_b200_basis_compute_jk); device pointers."""
        L = self.lib
        L.simint_b200_basis_compute_jk.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_void_p, C.c_longlong, C.c_void_p]
        r = L.simint_b200_basis_compute_jk(self.h, prec, C.c_void_p(dev_D), C.c_void_p(dev_J),
                                           C.c_void_p(dev_K), C.c_void_p(dev_scratch), scratch_doubles,
                                           C.c_void_p(stream))
        if r < 0:
            raise RuntimeError("simint_b200_basis_compute_jk failed: " + last_error())
        return r

    def class_times(self, prec, dev_ptr, ndoubles, stream=0):
        n = self.lib.simint_b200_basis_nclass(self.h)
        ms = (C.c_float * max(n, 1))()
        r = self.lib.simint_b200_basis_class_times(self.h, prec, C.c_void_p(dev_ptr), ndoubles,
                                                   C.c_void_p(stream), ms)
        if r < 0:
            raise RuntimeError("class_times failed: " + last_error())
        return list(ms)[:n]
