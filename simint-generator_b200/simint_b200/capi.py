"""ctypes mirror of the Simint C ABI (structs and prototypes).

The struct layouts follow include/simint/shell/shell.h, which keeps the
reference's field order (skel/simint/shell/shell.h:18-32, :47-85 with
SIMINT_OSTEI_MAXDER = 1).  The same definitions bind libsimint_b200.so, the
CPU oracle and the reference-built checker library.
"""

import ctypes as C

import numpy as np

SIMINT_SCREEN_NONE = 0
SIMINT_SCREEN_SCHWARZ = 1
SIMINT_SCREEN_FASTSCHWARZ = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class SimintShell(C.Structure):
    _fields_ = [("am", C.c_int), ("nprim", C.c_int),
                ("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("alpha", _dp), ("coef", _dp),
                ("memsize", C.c_size_t), ("ptr", C.c_void_p)]


class SimintMultiShellpair(C.Structure):
    _fields_ = [("am1", C.c_int), ("am2", C.c_int), ("nprim", C.c_int),
                ("nshell12", C.c_int), ("nshell12_clip", C.c_int),
                ("nprim12", _ip),
                ("AB_x", _dp), ("AB_y", _dp), ("AB_z", _dp),
                ("x", _dp), ("y", _dp), ("z", _dp),
                ("PA_x", _dp), ("PA_y", _dp), ("PA_z", _dp),
                ("PB_x", _dp), ("PB_y", _dp), ("PB_z", _dp),
                ("alpha", _dp), ("alpha2", _dp), ("beta2", _dp),
                ("prefac", _dp), ("screen", _dp), ("screen_max", C.c_double),
                ("memsize", C.c_size_t), ("ptr", C.c_void_p)]


ShellP = C.POINTER(SimintShell)
PairP = C.POINTER(SimintMultiShellpair)

PRIM_ARRAYS = ("x", "y", "z", "PA_x", "PA_y", "PA_z", "PB_x", "PB_y", "PB_z",
               "alpha", "alpha2", "beta2", "prefac", "screen")


def padded_nprim(pair):
    """Number of primitive slots including the 8-wide padding."""
    n, idx = pair.nshell12, 0
    for p in range(n):
        idx += pair.nprim12[p]
        if (p + 1) % 16 == 0 or p + 1 >= n:
            idx = (idx + 7) & ~7
    return idx


def pair_arrays(pair):
    """Copy every array of a multi-shell-pair into numpy (for comparisons)."""
    npad = padded_nprim(pair)
    out = {"am1": pair.am1, "am2": pair.am2, "nprim": pair.nprim,
           "nshell12": pair.nshell12, "nshell12_clip": pair.nshell12_clip,
           "screen_max": pair.screen_max}
    out["nprim12"] = np.ctypeslib.as_array(pair.nprim12, (pair.nshell12,)).copy()
    for k in ("AB_x", "AB_y", "AB_z"):
        out[k] = np.ctypeslib.as_array(getattr(pair, k), (pair.nshell12,)).copy()
    for k in PRIM_ARRAYS:
        ptr = getattr(pair, k)
        out[k] = None if not ptr else np.ctypeslib.as_array(ptr, (npad,)).copy()
    return out


def declare_shell_api(lib):
    """Attach argtypes/restype for the shell and pair functions."""
    V = None
    sigs = {
        "simint_initialize_shell": (V, [ShellP]),
        "simint_initialize_shells": (V, [C.c_int, ShellP]),
        "simint_allocate_shell": (V, [C.c_int, ShellP]),
        "simint_free_shell": (V, [ShellP]),
        "simint_free_shells": (V, [C.c_int, ShellP]),
        "simint_copy_shell": (V, [ShellP, ShellP]),
        "simint_normalize_shells": (V, [C.c_int, ShellP]),
        "simint_create_shell": (V, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    _dp, _dp, ShellP]),
        "simint_create_zero_shell": (V, [ShellP]),
        "simint_initialize_multi_shellpair": (V, [PairP]),
        "simint_initialize_multi_shellpairs": (V, [C.c_int, PairP]),
        "simint_allocate_multi_shellpair": (V, [C.c_int, ShellP, C.c_int, ShellP, PairP, C.c_int]),
        "simint_allocate_multi_shellpair2": (V, [C.c_int, ShellP, PairP, C.c_int]),
        "simint_free_multi_shellpair": (V, [PairP]),
        "simint_free_multi_shellpairs": (V, [C.c_int, PairP]),
        "simint_fill_multi_shellpair": (V, [C.c_int, ShellP, C.c_int, ShellP, PairP, C.c_int]),
        "simint_fill_multi_shellpair2": (V, [C.c_int, ShellP, PairP, C.c_int]),
        "simint_create_multi_shellpair": (V, [C.c_int, ShellP, C.c_int, ShellP, PairP, C.c_int]),
        "simint_create_multi_shellpair2": (V, [C.c_int, ShellP, PairP, C.c_int]),
        "simint_cat_multi_shellpair": (V, [C.c_int, C.POINTER(PairP), PairP, C.c_int]),
        "simint_cat_shellpairs": (V, [C.c_int, C.POINTER(PairP), PairP, C.c_int]),
        "simint_shellscreen": (C.c_double, [ShellP, ShellP, C.c_int]),
        "simint_primscreen": (C.c_double, [ShellP, ShellP, _dp, C.c_int]),
        "simint_shellscreen_schwarz": (C.c_double, [ShellP, ShellP]),
        "simint_shellscreen_fastschwarz": (C.c_double, [ShellP, ShellP]),
        "simint_primscreen_schwarz": (C.c_double, [ShellP, ShellP, _dp]),
        "simint_primscreen_fastschwarz": (C.c_double, [ShellP, ShellP, _dp]),
    }
    for name, (res, args) in sigs.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    return lib


class ShellSet:
    """A Python-owned array of simint_shell structs (alpha/coef kept alive).

    Shell i's storage is the numpy buffer kept in self._keep; ptr points at
    it, so compare_shell() recognises a pair of a shell with itself exactly
    as in C (same nprim and same ptr)."""

    def __init__(self, shells):
        # shells: list of (am, (x,y,z), alphas, coefs)
        self.n = len(shells)
        self.arr = (SimintShell * max(self.n, 1))()
        self._keep = []
        for i, (am, xyz, al, co) in enumerate(shells):
            buf = np.ascontiguousarray(np.concatenate([np.asarray(al, float), np.asarray(co, float)]))
            self._keep.append(buf)
            s = self.arr[i]
            s.am = int(am)
            s.nprim = len(al)
            s.x, s.y, s.z = (float(v) for v in xyz)
            s.alpha = buf.ctypes.data_as(_dp)
            s.coef = C.cast(buf.ctypes.data + 8 * len(al), _dp)
            s.memsize = buf.nbytes
            s.ptr = buf.ctypes.data

    def ptr(self, i=0):
        return C.cast(C.byref(self.arr, i * C.sizeof(SimintShell)), ShellP)

    def subset(self, idx):
        """Array of struct copies (sharing storage) for the listed shells."""
        out = (SimintShell * max(len(idx), 1))()
        for k, i in enumerate(idx):
            out[k] = self.arr[i]
        return out

    def pair_list(self, pairs):
        """2*npair array [A0 B0 A1 B1 ...] for simint_create_multi_shellpair2."""
        out = (SimintShell * max(2 * len(pairs), 1))()
        for k, (i, j) in enumerate(pairs):
            out[2 * k] = self.arr[i]
            out[2 * k + 1] = self.arr[j]
        return out

    def coefs(self, i):
        s = self.arr[i]
        return np.ctypeslib.as_array(s.coef, (s.nprim,)).copy()
