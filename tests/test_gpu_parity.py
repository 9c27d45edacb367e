"""GPU parity: libsimint_b200.so (through the C ABI) against the CPU oracle.

Every AM class up to (dd|dd) in both orderings, a sample of f and g classes,
screening on and off, multi-pair bra lists crossing the 16-pair padding
boundary, deriv=1.  The oracle builds its own pairs from the same shells;
the product builds them with simint_create_multi_shellpair2 (host code of
the library).  Bar: |d| <= 1e-13 or rel <= 1e-11 per element (FP64 path).
"""
import ctypes as C
import itertools

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from oracle import load_oracle
from _util import class_shells, oracle_pairs, oracle_eri, parity_bad

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def libs():
    lib = sb.load()
    lib.simint_init()
    return lib, load_oracle()


def _run_class(lib, orc, am, ordering, rng, deriv=0, nsh=(2, 1, 2, 1), tol=0.0, screen=0,
               nprim=(1, 3)):
    shells, grp = class_shells(rng, am, nsh=nsh, nprim=nprim)
    S = ShellSet(shells)
    orc.oracle_normalize_shells(S.n, S.ptr(0))
    bra = [(i, j) for i in grp[0] for j in grp[1]]
    ket = [(i, j) for i in grp[2] for j in grp[3]]
    lib.simint_b200_set_ordering(ordering)
    P = sb.make_pairs(lib, S, bra, screen)
    Q = sb.make_pairs(lib, S, ket, screen)
    r, out = sb.compute_eri(P, Q, tol, deriv, lib)
    oP = oracle_pairs(orc, S, bra, screen)
    oQ = oracle_pairs(orc, S, ket, screen)
    rr, ref = oracle_eri(orc, oP, oQ, tol, deriv, ordering)
    lib.simint_free_multi_shellpair(C.byref(P))
    lib.simint_free_multi_shellpair(C.byref(Q))
    orc.oracle_free_pair(C.byref(oP))
    orc.oracle_free_pair(C.byref(oQ))
    return r, rr, out, ref


CLASSES_D = list(itertools.product(range(3), repeat=4))


@pytest.mark.parametrize("ordering", [0, 1])
@pytest.mark.parametrize("am", CLASSES_D, ids=lambda a: "".join("spdfg"[x] for x in a))
def test_deriv0_upto_d(libs, am, ordering):
    lib, orc = libs
    rng = np.random.default_rng(hash(am) % 2**32 + 17 * ordering)
    r, rr, out, ref = _run_class(lib, orc, am, ordering, rng)
    assert r == rr
    bad, dmax = parity_bad(out, ref)
    assert len(bad) == 0, (am, dmax, out[bad[:5]], ref[bad[:5]])


@pytest.mark.parametrize("am", [(3, 0, 0, 0), (3, 1, 2, 0), (3, 3, 1, 1), (2, 3, 3, 2), (3, 3, 3, 3),
                                (4, 0, 0, 0), (4, 1, 3, 0), (0, 4, 4, 2), (4, 4, 4, 4), (1, 4, 2, 3)],
                         ids=lambda a: "".join("spdfg"[x] for x in a))
def test_deriv0_fg(libs, am):
    lib, orc = libs
    rng = np.random.default_rng(sum(am) * 31 + am[0])
    r, rr, out, ref = _run_class(lib, orc, am, 1, rng, nsh=(1, 1, 1, 1), nprim=(1, 2))
    assert r == rr
    bad, dmax = parity_bad(out, ref)
    assert len(bad) == 0, (am, dmax)


@pytest.mark.parametrize("am", [(0, 0, 0, 0), (1, 0, 1, 0), (1, 1, 1, 1), (2, 1, 0, 1), (2, 2, 2, 2),
                                (0, 2, 1, 2)], ids=lambda a: "".join("spdfg"[x] for x in a))
@pytest.mark.parametrize("ordering", [0, 1])
def test_deriv1(libs, am, ordering):
    lib, orc = libs
    rng = np.random.default_rng(7 + sum(am))
    r, rr, out, ref = _run_class(lib, orc, am, ordering, rng, deriv=1, nsh=(1, 2, 2, 1))
    assert r == rr
    bad, dmax = parity_bad(out, ref)
    assert len(bad) == 0, (am, dmax)


@pytest.mark.parametrize("screen", [1, 2])
@pytest.mark.parametrize("tol", [1e-14, 1e-10, 1e-6])
def test_screening_semantics(libs, screen, tol):
    """Primitive and 8-wide-vector screening skip exactly what the oracle skips."""
    lib, orc = libs
    rng = np.random.default_rng(int(tol * 1e16) % 1000 + screen)
    am = (1, 1, 1, 0)
    r, rr, out, ref = _run_class(lib, orc, am, 0, rng, nsh=(3, 2, 4, 5), tol=tol, screen=screen,
                                 nprim=(1, 4))
    assert r == rr
    if r > 0:
        bad, dmax = parity_bad(out, ref)
        assert len(bad) == 0, dmax


def test_many_bra_pairs_padding(libs):
    """More than 16 bra pairs: the padded offsets of later pairs are honoured."""
    lib, orc = libs
    rng = np.random.default_rng(99)
    r, rr, out, ref = _run_class(lib, orc, (1, 0, 1, 1), 0, rng, nsh=(9, 3, 2, 3), nprim=(1, 3))
    assert r == rr == 27 * 6
    bad, dmax = parity_bad(out, ref)
    assert len(bad) == 0, dmax


def test_ssss_clipped_ket_vector(libs):
    """(ss|ss) with a ket list clipped inside a vector: the reference's
    (ss|ss) kernel tests that vector with zeros past the clip
    (skel/ostei_s_s_s_s.c), so a vector whose only large screening values
    lie past the clip is skipped.  Ket pairs 0..4 tiny, 5..19 normal; clips
    5 (vector skipped: zeros), 7 and 20 (computed); the caller's pair data
    is left unchanged (the clip-20 call after the clip-5 one agrees with
    the oracle too)."""
    lib, orc = libs
    rng = np.random.default_rng(606)
    shells = [(0, tuple(rng.uniform(-1, 1, 3)), np.array([1.3]), np.array([0.8])),
              (0, tuple(rng.uniform(-1, 1, 3)), np.array([0.7]), np.array([0.9]))]
    for k in range(20):
        c = 1e-10 if k < 5 else 0.7
        for _ in range(2):
            shells.append((0, tuple(rng.uniform(-2, 2, 3)), np.array([rng.uniform(0.3, 3.0)]), np.array([c])))
    bra = [(0, 1)]
    ket = [(2 + 2 * k, 3 + 2 * k) for k in range(20)]
    S = ShellSet(shells)
    tol = 1e-6
    P = sb.make_pairs(lib, S, bra, 1)
    Q = sb.make_pairs(lib, S, ket, 1)
    oP = oracle_pairs(orc, S, bra, 1)
    oQ = oracle_pairs(orc, S, ket, 1)
    screen0 = np.ctypeslib.as_array(Q.screen, shape=(24,)).copy()
    try:
        for clip in (5, 20, 7, 5):
            Q.nshell12_clip = clip
            oQ.nshell12_clip = clip
            r, out = sb.compute_eri(P, Q, tol, 0, lib)
            rr, ref = oracle_eri(orc, oP, oQ, tol)
            assert r == rr == clip
            bad, dmax = parity_bad(out, ref)
            assert len(bad) == 0, (clip, dmax)
            if clip == 5:
                assert (out == 0).all()
            else:
                assert np.abs(out[5:]).max() > 1e-3
            assert np.array_equal(np.ctypeslib.as_array(Q.screen, shape=(24,)), screen0)
    finally:
        lib.simint_free_multi_shellpair(C.byref(P))
        lib.simint_free_multi_shellpair(C.byref(Q))
        orc.oracle_free_pair(C.byref(oP))
        orc.oracle_free_pair(C.byref(oQ))
