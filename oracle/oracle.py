"""ctypes loader for the CPU oracle and the reference-built checker library.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""

import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "simint-generator_b200"))

from simint_b200.capi import ShellP, PairP, declare_shell_api  # noqa: E402

_dp = C.POINTER(C.c_double)


def _recipe():
    """oracle/build.py, loaded by path (another build.py may be first on
    sys.path)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_build_recipe", os.path.join(HERE, "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def load_oracle():
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        _recipe().build_oracle()
        build_oracle()
    lib = C.CDLL(path)
    lib.oracle_create_pair.argtypes = [C.c_int, ShellP, PairP, C.c_int]
    lib.oracle_create_pair.restype = None
    lib.oracle_free_pair.argtypes = [PairP]
    lib.oracle_free_pair.restype = None
    lib.oracle_compute_eri.argtypes = [PairP, PairP, C.c_double, C.c_int, C.c_int, _dp]
    lib.oracle_compute_eri.restype = C.c_int
    lib.oracle_normalize_shells.argtypes = [C.c_int, ShellP]
    lib.oracle_normalize_shells.restype = None
    lib.oracle_boys.argtypes = [C.c_double, C.c_int, _dp]
    lib.oracle_boys.restype = None
    lib.oracle_count_primq.argtypes = [PairP, PairP, C.c_double]
    lib.oracle_count_primq.restype = C.c_longlong
    lib.oracle_shellscreen_schwarz.argtypes = [ShellP, ShellP]
    lib.oracle_shellscreen_schwarz.restype = C.c_double
    lib.oracle_bench_omp.argtypes = [C.c_int, PairP, PairP, C.c_double, C.c_int, C.c_int,
                                     C.c_int, _dp]
    lib.oracle_bench_omp.restype = C.c_double
    lib.oracle_bench_rows.argtypes = [C.c_int, C.POINTER(PairP), C.POINTER(PairP), C.c_double,
                                      C.c_int, C.POINTER(C.c_longlong), _dp]
    lib.oracle_bench_rows.restype = C.c_double
    lib.oracle_oei_st.argtypes = [C.c_int, ShellP, ShellP, _dp]
    lib.oracle_oei_st.restype = C.c_int
    lib.oracle_oei_potential.argtypes = [C.c_int, _dp, _dp, _dp, _dp, ShellP, ShellP, _dp]
    lib.oracle_oei_potential.restype = C.c_int
    return lib


def load_oracle_ld():
    """The oracle evaluated in long double (same pairs, same algorithm);
    oracle_compute_eri writes long double values."""
    path = os.path.join(HERE, "liboracle_ld.so")
    if not os.path.exists(path):
        _recipe().build_oracle_ld()
    lib = C.CDLL(path)
    lib.oracle_compute_eri.argtypes = [PairP, PairP, C.c_double, C.c_int, C.c_int, C.c_void_p]
    lib.oracle_compute_eri.restype = C.c_int
    # one-electron integrals: evaluated in long double, rounded to double
    lib.oracle_oei_st.argtypes = [C.c_int, ShellP, ShellP, _dp]
    lib.oracle_oei_st.restype = C.c_int
    lib.oracle_oei_potential.argtypes = [C.c_int, _dp, _dp, _dp, _dp, ShellP, ShellP, _dp]
    lib.oracle_oei_potential.restype = C.c_int
    return lib


def load_ref():
    """The reference-built library, or None when it was not built here."""
    path = os.path.join(HERE, "_ref", "libsimint_ref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    declare_shell_api(lib)
    lib.ref_valeev_integrals.argtypes = [ShellP, C.c_int, ShellP, C.c_int, ShellP, C.c_int,
                                         ShellP, C.c_int, _dp, C.c_int]
    lib.ref_valeev_integrals.restype = None
    lib.ref_boys_F.argtypes = [C.c_double, C.c_int, _dp]
    lib.ref_boys_F.restype = None
    lib.ref_boys_grid.argtypes = [C.c_int, C.c_int]
    lib.ref_boys_grid.restype = C.c_double
    lib.ref_boys_longfac.argtypes = [C.c_int]
    lib.ref_boys_longfac.restype = C.c_double
    for f in ("simint_compute_osoei_overlap", "simint_compute_osoei_ke"):
        getattr(lib, f).argtypes = [ShellP, ShellP, _dp]
        getattr(lib, f).restype = C.c_int
    lib.simint_compute_osoei_potential.argtypes = [C.c_int, _dp, _dp, _dp, _dp, ShellP, ShellP, _dp]
    lib.simint_compute_osoei_potential.restype = C.c_int
    return lib
