"""Shared helpers for the tests (parity comparisons and shell sets)."""
import ctypes as C
import itertools

import numpy as np

from simint_b200.capi import ShellSet, SimintMultiShellpair, ShellP
from simint_b200.workloads import random_shells

NC = lambda l: (l + 1) * (l + 2) // 2

# Parity bar of the FP64 path against the CPU oracle, per element:
# |d| <= 1e-13, or |ref| > 1e-15 and |d|/|ref| <= 1e-11.
ABS_TOL = 1e-13
REL_TOL = 1e-11


def parity_bad(calc, ref, abs_tol=ABS_TOL, rel_tol=REL_TOL):
    """Indices failing the abs-or-rel bar."""
    d = np.abs(calc - ref)
    rel = np.where(np.abs(ref) > 1e-15, d / np.maximum(np.abs(ref), 1e-300), np.inf)
    bad = (d > abs_tol) & ~(rel <= rel_tol)
    return np.nonzero(bad)[0], d.max() if d.size else 0.0


def class_shells(rng, am, nsh=(2, 1, 2, 1), nprim=(1, 3), alpha=(0.1, 20.0), box=3.0):
    ams = [am[0]] * nsh[0] + [am[1]] * nsh[1] + [am[2]] * nsh[2] + [am[3]] * nsh[3]
    shells = random_shells(rng, ams, nprim_range=nprim, alpha=alpha, box=box)
    idx = np.cumsum([0] + list(nsh))
    grp = [list(range(idx[k], idx[k + 1])) for k in range(4)]
    return shells, grp


def oracle_pairs(orc, S, pairs, screen=0):
    P = SimintMultiShellpair()
    arr = S.pair_list(pairs)
    orc.oracle_create_pair(len(pairs), C.cast(arr, ShellP), C.byref(P), screen)
    return P


def oracle_eri(orc, P, Q, tol=0.0, deriv=0, ordering=0):
    n = P.nshell12_clip * Q.nshell12_clip * NC(P.am1) * NC(P.am2) * NC(Q.am1) * NC(Q.am2)
    out = np.zeros(n * (12 if deriv else 1))
    r = orc.oracle_compute_eri(C.byref(P), C.byref(Q), tol, deriv, ordering,
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    return r, out


def oracle_eri_ld(orc_ld, P, Q, tol=0.0, deriv=0, ordering=0):
    """The same integrals from the long-double build of the oracle."""
    n = P.nshell12_clip * Q.nshell12_clip * NC(P.am1) * NC(P.am2) * NC(Q.am1) * NC(Q.am2)
    out = np.zeros(n * (12 if deriv else 1), dtype=np.longdouble)
    r = orc_ld.oracle_compute_eri(C.byref(P), C.byref(Q), tol, deriv, ordering, out.ctypes.data)
    return r, out


def as_accurate_as_oracle(calc, ref, ref_ld, slack=2.0, floor=1e-14):
    """Indices where calc is further from the long-double values than
    slack x the double-precision oracle's largest error over the same block
    (plus floor): the elements on which calc is less accurate than the
    reference algorithm evaluated in double."""
    e_calc = np.abs(calc.astype(np.longdouble) - ref_ld)
    e_ref = float(np.abs(ref.astype(np.longdouble) - ref_ld).max()) if ref.size else 0.0
    return np.nonzero(e_calc > slack * e_ref + floor)[0]


def oracle_oei(orc, kind, S, a, b, centres=None):
    """One-electron integrals of shells a, b of S from the oracle: kind 0
    overlap, 1 kinetic energy, 2 nuclear attraction over centres (rows
    x, y, z, Z)."""
    dp = C.POINTER(C.c_double)
    out = np.zeros(NC(S.arr[a].am) * NC(S.arr[b].am))
    if kind < 2:
        r = orc.oracle_oei_st(kind, S.ptr(a), S.ptr(b), out.ctypes.data_as(dp))
    else:
        c = np.ascontiguousarray(np.asarray(centres, float).T)
        r = orc.oracle_oei_potential(c.shape[1], c[3].ctypes.data_as(dp), c[0].ctypes.data_as(dp),
                                     c[1].ctypes.data_as(dp), c[2].ctypes.data_as(dp),
                                     S.ptr(a), S.ptr(b), out.ctypes.data_as(dp))
    assert r == 1
    return out


def quartets_unexplained(calc, ref, ref_ld_of, nout, abs_tol=ABS_TOL, rel_tol=REL_TOL,
                         slack=2.0, floor=1e-14):
    """Quartets (blocks of nout elements) where calc misses the FP64 bar
    against ref AND is further from a long-double evaluation of the same
    quartet than slack x ref's own largest distance from it (+ floor).

    Two correct FP64 evaluations of an ill-conditioned quartet (exponents
    orders of magnitude apart on distant centres: the recurrences cancel)
    can differ far beyond the bar -- the reference's default and all-inline
    builds do, on about 1 quartet in 1e5 of the l <= 3 workload.  Such a
    quartet passes when calc is as close to the long-double values as the
    reference is.  ref_ld_of(q) returns the long-double values of quartet q.
    Returns (unexplained quartet indices, number outside the bar)."""
    c = calc.reshape(-1, nout)
    r = ref.reshape(-1, nout)
    d = np.abs(c - r)
    rel = np.where(np.abs(r) > 1e-15, d / np.maximum(np.abs(r), 1e-300), np.inf)
    outq = np.nonzero(((d > abs_tol) & ~(rel <= rel_tol)).any(axis=1))[0]
    bad = []
    for q in outq:
        ld = np.asarray(ref_ld_of(int(q)), dtype=np.longdouble)
        e_c = float(np.abs(c[q].astype(np.longdouble) - ld).max())
        e_r = float(np.abs(r[q].astype(np.longdouble) - ld).max())
        if e_c > slack * e_r + floor:
            bad.append((int(q), e_c, e_r))
    return bad, len(outq)


class RowLD:
    """Long-double evaluations (oracle/liboracle_ld.so) of single quartets
    (bra pair, ket pair) of a shell list, built with the oracle's own pair
    code and primitive screening."""

    def __init__(self, orc, orc_ld, shells, screen=0, tol=0.0, deriv=0, ordering=0,
                 normalize=True):
        self.orc, self.orc_ld = orc, orc_ld
        self.S = ShellSet(shells)
        if normalize:
            orc.oracle_normalize_shells(self.S.n, self.S.ptr(0))
        self.screen, self.tol, self.deriv, self.ordering = screen, tol, deriv, ordering

    def __call__(self, bra, ket):
        P = oracle_pairs(self.orc, self.S, [bra], self.screen)
        Q = oracle_pairs(self.orc, self.S, [ket], self.screen)
        r, out = oracle_eri_ld(self.orc_ld, P, Q, self.tol, self.deriv, self.ordering)
        self.orc.oracle_free_pair(C.byref(P))
        self.orc.oracle_free_pair(C.byref(Q))
        return out


def in_child_process(fn):
    """Run a test in a child pytest process (the same test id), so that a
    crash of the process -- these tests drive both libraries from 16 OpenMP
    threads of a C driver -- fails that test alone instead of ending the
    whole session.  The child runs the body itself (SB_TEST_CHILD=1)."""
    import functools
    import os
    import subprocess
    import sys

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        if os.environ.get("SB_TEST_CHILD") == "1":
            return fn(*args, **kwargs)
        node = os.environ.get("PYTEST_CURRENT_TEST", "").rsplit(" ", 1)[0]
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        env = dict(os.environ, SB_TEST_CHILD="1")
        r = subprocess.run([sys.executable, "-m", "pytest", node, "-q", "-p", "no:cacheprovider", "-x"],
                           cwd=root, env=env, capture_output=True, text=True, timeout=1500)
        out = (r.stdout + r.stderr)[-4000:]
        assert r.returncode == 0, "child pytest for %s ended with %d:\n%s" % (node, r.returncode, out)
    return wrapper
