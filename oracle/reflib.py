"""ctypes access to the reference's generated CPU library (oracle/_ref/).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's reference arm / cpu_baseline leg, never by the product.

The libraries are built by oracle/build_reflib.py (create.py output + the
reference runtime + oracle/refdrv.c).  `load(variant)` picks the AVX-512 build
when the host CPU has avx512f, else the AVX2 build; it raises FileNotFoundError
when the variant was not built.

RefLib wraps refdrv.c:
  set_shells(shells)            shells = [(am, (x, y, z), alpha[], coef[])]
  coefs()                       normalised coefficients (concatenated)
  schwarz(pairs)                max |(ab|ab)| per shell pair
  pairset(pairs, screen)        one multi shell pair over the pair list
  pairsets_single(pairs, screen)  one single-pair set per pair
  rows(bh, kh, kc, deriv, tol, threads, out=None)  simint_compute_eri_deriv per row
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")

_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_longlong)


def host_isa():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = line.split()
                    return "avx512" if ("avx512f" in fl and "avx512cd" in fl) else "avx2"
    except OSError:
        pass
    return "avx2"


def lib_path(variant, isa=None):
    return os.path.join(REF, "libsimint_%s_%s.so" % (variant, isa or host_isa()))


def available(variant, isa=None):
    return os.path.exists(lib_path(variant, isa))


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class RefLib:
    def __init__(self, path):
        self.path = path
        self.lib = C.CDLL(path)
        L = self.lib
        L.rd_init.restype = None
        L.rd_simd_len.restype = C.c_int
        L.rd_max_am.restype = C.c_int
        L.rd_max_der.restype = C.c_int
        L.rd_set_shells.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_int]
        L.rd_get_coefs.argtypes = [_dp]
        L.rd_get_coefs.restype = None
        L.rd_shell_schwarz.argtypes = [C.c_int, _ip, _dp, C.c_int]
        L.rd_shell_schwarz.restype = None
        L.rd_pairset.argtypes = [C.c_int, _ip, C.c_int]
        L.rd_pairsets_single.argtypes = [C.c_int, _ip, C.c_int, C.c_int]
        L.rd_pairsets_multi.argtypes = [C.c_int, _ip, _ip, C.c_int, C.c_int]
        L.rd_pairsets_free.restype = None
        L.rd_pairset_info.argtypes = [C.c_int, _ip, _ip, _dp]
        L.rd_rows.argtypes = [C.c_int, _ip, _ip, _ip, C.c_int, C.c_double, C.c_int, _dp, _lp,
                              _ip, _lp]
        L.rd_rows.restype = C.c_double
        L.rd_init()
        self.simd_len = L.rd_simd_len()
        self.max_am = L.rd_max_am()
        self.max_der = L.rd_max_der()
        self.nprim_total = 0

    def set_shells(self, shells, normalize=True):
        am = _arr([s[0] for s in shells], np.int32)
        npr = _arr([len(s[2]) for s in shells], np.int32)
        xyz = _arr([c for s in shells for c in s[1]], np.float64)
        al = _arr(np.concatenate([np.asarray(s[2], float) for s in shells]), np.float64)
        co = _arr(np.concatenate([np.asarray(s[3], float) for s in shells]), np.float64)
        self._keep = (am, npr, xyz, al, co)
        self.nprim_total = int(npr.sum())
        r = self.lib.rd_set_shells(len(shells), am.ctypes.data_as(_ip), npr.ctypes.data_as(_ip),
                                   xyz.ctypes.data_as(_dp), al.ctypes.data_as(_dp),
                                   co.ctypes.data_as(_dp), 1 if normalize else 0)
        if r != 0:
            raise MemoryError("rd_set_shells")

    def coefs(self):
        out = np.empty(self.nprim_total)
        self.lib.rd_get_coefs(out.ctypes.data_as(_dp))
        return out

    def schwarz(self, pairs, threads=None):
        p = _arr(pairs, np.int32).reshape(-1, 2)
        out = np.empty(len(p))
        self.lib.rd_shell_schwarz(len(p), p.ctypes.data_as(_ip), out.ctypes.data_as(_dp),
                                  threads or os.cpu_count() or 1)
        return out

    def pairset(self, pairs, screen=0):
        p = _arr(pairs, np.int32).reshape(-1, 2)
        h = self.lib.rd_pairset(len(p), p.ctypes.data_as(_ip), screen)
        if h < 0:
            raise MemoryError("rd_pairset")
        return h

    def pairsets_single(self, pairs, screen=0, threads=None):
        p = _arr(pairs, np.int32).reshape(-1, 2)
        h = self.lib.rd_pairsets_single(len(p), p.ctypes.data_as(_ip), screen,
                                        threads or os.cpu_count() or 1)
        if h < 0:
            raise MemoryError("rd_pairsets_single")
        return np.arange(h, h + len(p), dtype=np.int32)

    def pairsets_multi(self, sets, screen=0, threads=None):
        """One pair set per list in `sets`, built in parallel; handles."""
        counts = _arr([len(s) for s in sets], np.int32)
        p = _arr(np.concatenate([np.asarray(s, np.int32).reshape(-1, 2) for s in sets]), np.int32)
        h = self.lib.rd_pairsets_multi(len(sets), counts.ctypes.data_as(_ip), p.ctypes.data_as(_ip),
                                       screen, threads or os.cpu_count() or 1)
        if h < 0:
            raise MemoryError("rd_pairsets_multi")
        return list(range(h, h + len(sets)))

    def free_pairsets(self):
        self.lib.rd_pairsets_free()

    def pairset_info(self, h):
        n, npr, sm = C.c_int(), C.c_int(), C.c_double()
        self.lib.rd_pairset_info(h, C.byref(n), C.byref(npr), C.byref(sm))
        return n.value, npr.value, sm.value

    def rows(self, bh, kh, kc, deriv, tol, threads=None, out=None, off=None, count=True):
        """Returns (seconds, ret[], primq[])."""
        bh = _arr(bh, np.int32)
        kh = _arr(kh, np.int32)
        kc = _arr(kc, np.int32)
        n = len(bh)
        ret = np.zeros(n, np.int32)
        prq = np.zeros(n, np.int64) if count else None
        offa = _arr(off, np.int64) if off is not None else None
        t = self.lib.rd_rows(n, bh.ctypes.data_as(_ip), kh.ctypes.data_as(_ip),
                             kc.ctypes.data_as(_ip), deriv, tol, threads or os.cpu_count() or 1,
                             out.ctypes.data_as(_dp) if out is not None else None,
                             offa.ctypes.data_as(_lp) if offa is not None else None,
                             ret.ctypes.data_as(_ip),
                             prq.ctypes.data_as(_lp) if prq is not None else None)
        return t, ret, prq


_cache = {}


def load(variant, isa=None):
    path = lib_path(variant, isa)
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    _cache[path] = RefLib(path)
    return _cache[path]
