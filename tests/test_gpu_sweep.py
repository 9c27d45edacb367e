"""GPU: the batched, screened sweep (simint_b200_basis_*) against the oracle.

A small basis (s..g shells on a few pseudo-atoms) is swept in full-layout
mode.  For every row of every class (a bra pair against a prefix of the
class's ket list, stored by decreasing Schwarz bound) the oracle runs the
same call -- the whole ket list clipped to the row, the same primitive
Schwarz screening -- and every quartet the sweep kept is compared with it (bar: abs 1e-13 or rel 1e-11; a quartet with elements
outside it passes only if none of its elements is further from the
long-double evaluation of the same algorithm than twice the double-precision
oracle's largest error on that quartet, i.e. the gap is the intrinsic error
of the recurrences in double).  Checksums must equal sums over the
output; graph replay and streaming through a small buffer must reproduce
them."""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells
from oracle import load_oracle, load_oracle_ld
from _util import oracle_pairs, oracle_eri, oracle_eri_ld, parity_bad, as_accurate_as_oracle, NC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    orc = load_oracle()
    orc_ld = load_oracle_ld()
    rng = np.random.default_rng(2024)
    shells = random_shells(rng, [0, 0, 1, 1, 2, 3, 0, 1, 2, 0, 1, 4], nprim_range=(1, 4),
                           alpha=(0.1, 300.0), box=6.0, natom=4)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    return torch, lib, orc, orc_ld, S, [s[0] for s in shells]


def pair_class_list(ams, la, lb):
    ia = [i for i, a in enumerate(ams) if a == la]
    ib = [i for i, a in enumerate(ams) if a == lb]
    return [(i, j) for i in ia for j in ib if not (la == lb and j > i)]


@pytest.mark.parametrize("tol", [0.0, 1e-12])
@pytest.mark.parametrize("ordering", [0, 1])
def test_sweep_matches_oracle(setup, tol, ordering):
    torch, lib, orc, orc_ld, S, ams = setup
    lib.simint_b200_set_ordering(ordering)
    B = sb.Basis(S, tol, max_am=4, lib=lib)
    n = B.output_size
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    B.compute(sb.FP64, out.data_ptr(), n)
    torch.cuda.synchronize()
    host = out.cpu().numpy()
    sums = B.checksums()
    screen = 1 if tol > 0 else 0
    for k, c in enumerate(B.classes()):
        blk = host[c["offset"]:c["offset"] + c["nquart"] * c["nout"]]
        assert np.isclose(sums[k, 0], blk.sum(), rtol=1e-9, atol=1e-9)
        assert np.isclose(sums[k, 1], np.abs(blk).sum(), rtol=1e-9)
        # the rows of the class: one bra pair against a prefix of the ket
        # list in the sweep's stored order (decreasing Schwarz bound); the
        # oracle gets the same calls (the whole list, clipped to the row)
        kl = [tuple(int(x) for x in p) for p in B.class_kets(k)]
        Q = oracle_pairs(orc, S, kl, screen)
        sh4 = B.class_quartets(k, c["nquart"])
        for first, cnt in B.rows(k):
            a, b = (int(x) for x in sh4[first, :2])
            assert [tuple(x) for x in sh4[first:first + cnt, 2:]] == kl[:cnt]
            P = oracle_pairs(orc, S, [(a, b)], screen)
            Q.nshell12_clip = cnt
            r, ref = oracle_eri(orc, P, Q, tol, 0, ordering)
            orc.oracle_free_pair(C.byref(P))
            if r < 0:
                ref = np.zeros_like(ref)
            ref = ref.reshape(cnt, c["nout"])
            for i in range(cnt):
                q = first + i
                want = ref[i]
                got = blk[q * c["nout"]:(q + 1) * c["nout"]]
                bad, dmax = parity_bad(got, want)
                if len(bad):
                    # elements outside the abs/rel bar: the recurrences compute
                    # them with cancellation, so every double-precision
                    # evaluation has errors of that size; accept them only where
                    # the product is as close to the long-double evaluation as
                    # the oracle is
                    cc, d = kl[i]
                    P1 = oracle_pairs(orc, S, [(a, b)], screen)
                    Q1 = oracle_pairs(orc, S, [(cc, d)], screen)
                    _, want_ld = oracle_eri_ld(orc_ld, P1, Q1, tol, 0, ordering)
                    orc.oracle_free_pair(C.byref(P1))
                    orc.oracle_free_pair(C.byref(Q1))
                    worse = as_accurate_as_oracle(got, want, want_ld)
                    assert len(worse) == 0, (c["am"], q, dmax, got[worse[:4]], want[worse[:4]],
                                             np.abs(want).max())
        Q.nshell12_clip = len(kl)
        orc.oracle_free_pair(C.byref(Q))
    # graph replay gives the same checksums
    B.compute(sb.FP64, out.data_ptr(), n)
    B.compute(sb.FP64, out.data_ptr(), n)
    torch.cuda.synchronize()
    assert np.allclose(B.checksums(), sums, rtol=1e-9, atol=1e-12)
    # streamed through a small buffer: same checksums
    small = torch.empty(4096, dtype=torch.float64, device="cuda")
    B.compute(sb.FP64, small.data_ptr(), 4096)
    torch.cuda.synchronize()
    assert np.allclose(B.checksums(), sums, rtol=1e-9, atol=1e-12)
    B.close()
