"""GPU: large simint_compute_eri calls (>= 16 MB of output, >= 64 ket pairs)
take the chunked, pipelined path; results must meet the parity bar against
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
