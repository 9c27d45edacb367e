"""Pin the CPU oracle (and our host pair code) to the reference itself.

Golden fixtures in tests/golden were produced by tests/golden/make_golden.py
from libraries compiled from the reference's own sources: ValeevRef (the
long-double oracle of the reference's test_eri / test_eri_deriv1), the
reference's Boys function and its pair code (shell.c).  These tests run on
CPU only.
"""
import ctypes as C
import os

import numpy as np
import pytest

from simint_b200.capi import ShellSet, SimintMultiShellpair, ShellP, pair_arrays
from oracle import load_oracle
from _util import oracle_pairs, oracle_eri, parity_bad

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden(name):
    return np.load(os.path.join(GOLD, name))


def _classes(data):
    return sorted({k.split("/")[0] for k in data.files})


def _shells(data, key):
    am, xyz, nprim = data[key + "/am"], data[key + "/xyz"], data[key + "/nprim"]
    al, co = data[key + "/alpha"], data[key + "/coef"]
    out, o = [], 0
    for s in range(len(am)):
        n = int(nprim[s])
        out.append((int(am[s]), tuple(xyz[s]), al[o:o + n], co[o:o + n]))
        o += n
    return out


@pytest.fixture(scope="module")
def orc():
    return load_oracle()


def _oracle_vs_valeev(orc, data, key, deriv):
    shells = _shells(data, key)
    nsh = [int(x) for x in data[key + "/nsh"]]
    S = ShellSet(shells)   # coefficients already normalised
    idx = np.cumsum([0] + nsh)
    grp = [list(range(idx[k], idx[k + 1])) for k in range(4)]
    P = oracle_pairs(orc, S, [(i, j) for i in grp[0] for j in grp[1]])
    Q = oracle_pairs(orc, S, [(i, j) for i in grp[2] for j in grp[3]])
    r, out = oracle_eri(orc, P, Q, 0.0, deriv, 0)
    orc.oracle_free_pair(C.byref(P))
    orc.oracle_free_pair(C.byref(Q))
    return out, data[key + "/values"]


D0 = _golden("valeev_deriv0.npz")
D1 = _golden("valeev_deriv1.npz")


@pytest.mark.parametrize("key", _classes(D0))
def test_oracle_matches_valeevref_deriv0(orc, key):
    """The reference's own acceptance rule (test_eri.cpp:227): fail only if
    abs > 1e-14 and rel > 1e-8 (rel counted where |ref| > 1e-15)."""
    out, ref = _oracle_vs_valeev(orc, D0, key, 0)
    bad, dmax = parity_bad(out, ref, abs_tol=1e-14, rel_tol=1e-8)
    assert len(bad) == 0, (key, dmax)


@pytest.mark.parametrize("key", _classes(D1))
def test_oracle_matches_valeevref_deriv1(orc, key):
    """test_eri_deriv1.cpp:229 applies the same rule to the 12 components."""
    out, ref = _oracle_vs_valeev(orc, D1, key, 1)
    bad, dmax = parity_bad(out, ref, abs_tol=1e-14, rel_tol=1e-8)
    assert len(bad) == 0, (key, dmax)


def test_boys_grid_equals_reference_table():
    """Our mpmath-generated grid equals the reference's boys_shortgrid and
    boys_longfac (both correctly rounded values of the same function)."""
    from simint_b200.gen.boysgrid import make_table
    g = _golden("boys_ref.npz")
    rows, longfac = make_table()
    rows = np.array(rows)
    rel = np.abs(rows - g["grid"]) / np.abs(g["grid"])
    assert rel.max() <= 2.3e-16
    assert np.array_equal(np.array(longfac), g["longfac"])


def test_boys_evaluation_matches_reference(orc):
    g = _golden("boys_ref.npz")
    buf = np.zeros(40)
    for a, x in enumerate(g["x"]):
        for n in (0, 1, 2, 3, 4, 7, 12, 16):
            orc.oracle_boys(float(x), n, buf.ctypes.data_as(C.POINTER(C.c_double)))
            ref = g["F"][a, n, :n + 1]
            rel = np.abs(buf[:n + 1] - ref) / np.maximum(np.abs(ref), 1e-300)
            assert rel.max() <= 1e-13, (x, n, rel.max())


def test_boys_against_mpmath(orc):
    """Independent check against mpmath (30 digits).

    Below 36.5 the Taylor grid is accurate to ~1e-15.  At and above 36.5 the
    reference's scheme uses the asymptotic form F_n ~ (2n-1)!!/2^(n+1)
    sqrt(pi/x^(2n+1)) (boys_long.h:14-58) -- for the top order only when
    L >= 4, followed by downward recursion, which keeps the relative error --
    so the error there is the asymptotic remainder
    e^-x x^(n-1/2) / Gamma(n+1/2) of the highest order evaluated.  The
    reference carries this error too (up to ~1e-6 relative for L = 12 at
    x = 36.5); we reproduce its algorithm, not a more accurate one."""
    import mpmath as mp
    mp.mp.dps = 30
    buf = np.zeros(40)
    for L in (3, 12):
        for x in (0.0, 0.037, 1.234, 7.77, 20.05, 36.49, 36.5, 44.0, 90.0):
            orc.oracle_boys(x, L, buf.ctypes.data_as(C.POINTER(C.c_double)))
            for n in range(L + 1):
                exact = (mp.mpf(1) / (2 * n + 1)) if x == 0 else \
                    mp.gammainc(n + mp.mpf(1) / 2, 0, x) / (2 * mp.power(x, n + mp.mpf(1) / 2))
                tol = 1e-14
                if x >= 36.5:
                    top = L if L >= 4 else n
                    tol += 2 * float(mp.exp(-x) * mp.power(x, top - 0.5) / mp.gamma(top + 0.5))
                assert abs(buf[n] - float(exact)) <= tol * abs(float(exact)), (x, L, n)


PAIRS = _golden("pairs_ref.npz")


def _pair_shells():
    return _shells(PAIRS, "shells")


@pytest.mark.parametrize("name", ["mixed_0", "mixed_2", "self_0", "self_2"])
def test_oracle_pairs_match_reference_shell_c(orc, name):
    S = ShellSet(_pair_shells())
    pl = [tuple(p) for p in PAIRS[name + "/pairs"]]
    screen = int(name.split("_")[1])
    P = oracle_pairs(orc, S, pl, screen)
    a = pair_arrays(P)
    for k in ("nprim12", "AB_x", "x", "PA_y", "PB_z", "alpha", "alpha2", "beta2", "prefac"):
        np.testing.assert_array_equal(a[k], PAIRS[name + "/" + k], err_msg=k)
    if screen:
        np.testing.assert_allclose(a["screen"], PAIRS[name + "/screen"], rtol=1e-15)
    orc.oracle_free_pair(C.byref(P))


@pytest.mark.parametrize("name", ["mixed_0", "mixed_2", "self_0", "self_2"])
def test_library_pairs_match_reference_shell_c(name):
    """libsimint_b200's host pair code reproduces shell.c bit for bit
    (no screening and fast-Schwarz screening need no GPU)."""
    import simint_b200 as sb
    lib = sb.load()
    S = ShellSet(_pair_shells())
    pl = [tuple(p) for p in PAIRS[name + "/pairs"]]
    screen = int(name.split("_")[1])
    P = sb.make_pairs(lib, S, pl, screen)
    a = pair_arrays(P)
    for k in ("nprim12", "AB_x", "AB_y", "AB_z", "x", "y", "z", "PA_x", "PA_y", "PA_z",
              "PB_x", "PB_y", "PB_z", "alpha", "alpha2", "beta2", "prefac"):
        np.testing.assert_array_equal(a[k], PAIRS[name + "/" + k], err_msg=k)
    assert a["nprim"] == int(PAIRS[name + "/nprim"])
    assert a["nshell12"] == len(pl)
    if screen:
        np.testing.assert_allclose(a["screen"], PAIRS[name + "/screen"], rtol=1e-15)
    lib.simint_free_multi_shellpair(C.byref(P))


@pytest.mark.parametrize("key", _classes(D0)[::4])
def test_long_double_oracle_against_valeevref(orc, key):
    """The long-double build of the oracle (used to measure the intrinsic
    double-precision error of cancelling elements) is at least as close to
    ValeevRef (the reference's long-double oracle) as the double build."""
    from oracle import load_oracle_ld
    from _util import oracle_eri_ld
    orc_ld = load_oracle_ld()
    shells = _shells(D0, key)
    nsh = [int(x) for x in D0[key + "/nsh"]]
    S = ShellSet(shells)
    idx = np.cumsum([0] + nsh)
    grp = [list(range(idx[k], idx[k + 1])) for k in range(4)]
    P = oracle_pairs(orc, S, [(i, j) for i in grp[0] for j in grp[1]])
    Q = oracle_pairs(orc, S, [(i, j) for i in grp[2] for j in grp[3]])
    _, out = oracle_eri(orc, P, Q, 0.0, 0, 0)
    _, out_ld = oracle_eri_ld(orc_ld, P, Q, 0.0, 0, 0)
    orc.oracle_free_pair(C.byref(P))
    orc.oracle_free_pair(C.byref(Q))
    ref = D0[key + "/values"].astype(np.longdouble)
    e64 = float(np.abs(out - ref).max())
    eld = float(np.abs(out_ld - ref).max())
    scale = float(np.abs(ref).max())
    assert eld <= e64 + 2e-16 * scale, (key, eld, e64)


OEI = _golden("oei_ref.npz")


@pytest.mark.parametrize("key", _classes(OEI))
def test_oracle_one_electron_matches_reference(orc, key):
    """Overlap, kinetic energy and nuclear attraction of the oracle against
    the reference's own osoei code (skel/simint/osoei) on the same shells:
    within 1e-14 of the block's largest value (the two evaluations differ
    only in recursion direction and rounding)."""
    from _util import oracle_oei
    S = ShellSet(_shells(OEI, key))
    cen = OEI[key + "/centres"]
    ref = OEI[key + "/values"]
    for kind in range(3):
        for a in range(2):
            for b in range(2):
                out = oracle_oei(orc, kind, S, a, 2 + b, cen)
                r = ref[kind, a, b]
                scale = max(1.0, float(np.abs(r).max()))
                assert np.abs(out - r).max() <= 1e-14 * scale, (key, kind, a, b, np.abs(out - r).max())
