"""GPU: large simint_compute_eri calls (>= 16 MB moved: results plus ket
pair records; >= 64 ket pairs) take the chunked, pipelined path; results must meet the parity bar against
the oracle for one and several bra pairs, with and without screening, and
the return value must be the reference's."""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells
from oracle import load_oracle
from _util import oracle_pairs, oracle_eri, parity_bad

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nbra,screen,tol", [(1, 0, 0.0), (3, 1, 1e-12)], ids=["one_bra", "three_bra_screened"])
def test_pipelined_call_matches_oracle(nbra, screen, tol):
    lib = sb.load()
    lib.simint_init()
    lib.simint_b200_set_ordering(0)
    orc = load_oracle()
    rng = np.random.default_rng(321 + nbra)
    am = (2, 2, 2, 1)
    nk1, nk2 = 80, 60
    ams = [am[0]] * nbra + [am[1]] + [am[2]] * nk1 + [am[3]] * nk2
    S = ShellSet(random_shells(rng, ams, nprim_range=(1, 2), alpha=(0.3, 30.0), box=8.0, natom=12))
    orc.oracle_normalize_shells(S.n, S.ptr(0))
    bra = [(i, nbra) for i in range(nbra)]
    o = nbra + 1
    ket = [(o + i, o + nk1 + j) for i in range(nk1) for j in range(nk2)]
    P = sb.make_pairs(lib, S, bra, screen)
    Q = sb.make_pairs(lib, S, ket, screen)
    nout = 6 * 6 * 6 * 3
    assert len(bra) * len(ket) * nout * 8 >= 16 << 20
    r, out = sb.compute_eri(P, Q, tol, 0, lib)
    oP, oQ = oracle_pairs(orc, S, bra, screen), oracle_pairs(orc, S, ket, screen)
    rr, ref = oracle_eri(orc, oP, oQ, tol, 0, 0)
    assert r == rr
    bad, dmax = parity_bad(out, ref)
    assert len(bad) == 0, dmax
    for X in (P, Q):
        lib.simint_free_multi_shellpair(C.byref(X))
    for X in (oP, oQ):
        orc.oracle_free_pair(C.byref(X))


def test_upload_heavy_call_matches_oracle():
    """A long ket list of a small class: little output (0.6 MB) but about
    25 MB of ket records, so the call is pipelined on its uploads."""
    lib = sb.load()
    lib.simint_init()
    lib.simint_b200_set_ordering(0)
    orc = load_oracle()
    rng = np.random.default_rng(77)
    nk1, nk2 = 90, 90
    ams = [1, 0] + [1] * nk1 + [0] * nk2
    S = ShellSet(random_shells(rng, ams, nprim_range=(4, 6), alpha=(0.2, 40.0), box=10.0, natom=30))
    orc.oracle_normalize_shells(S.n, S.ptr(0))
    bra = [(0, 1)]
    ket = [(2 + i, 2 + nk1 + j) for i in range(nk1) for j in range(nk2)]
    P = sb.make_pairs(lib, S, bra, 1)
    Q = sb.make_pairs(lib, S, ket, 1)
    assert Q.nprim * 16 * 8 >= 16 << 20
    r, out = sb.compute_eri(P, Q, 1e-12, 0, lib)
    oP, oQ = oracle_pairs(orc, S, bra, 1), oracle_pairs(orc, S, ket, 1)
    rr, ref = oracle_eri(orc, oP, oQ, 1e-12, 0, 0)
    assert r == rr
    bad, dmax = parity_bad(out, ref)
    assert len(bad) == 0, dmax
    for X in (P, Q):
        lib.simint_free_multi_shellpair(C.byref(X))
    for X in (oP, oQ):
        orc.oracle_free_pair(C.byref(X))
