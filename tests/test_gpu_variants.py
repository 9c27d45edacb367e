"""GPU: every kernel variant of a class against the CPU oracle.

The autotuner may pick, per class, the register kernel, the cooperative
kernel with 256, 128 or 64 threads and 1, 2, 4 or 8 primitive quartets per
wavefront pass, the column kernel with 4 or 8 primitive quartets per batch (83: 4 in two thread groups per CTA),
the first cooperative kernel or the generic kernel; each must meet the FP64
parity bar on its own.  Variants are pinned with simint_b200_set_variant and restored
to the default rule afterwards.
"""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from oracle import load_oracle
from _util import class_shells, oracle_pairs, oracle_eri, parity_bad

pytestmark = pytest.mark.gpu

VARIANTS = [sb.VAR_STRAIGHT, sb.VAR_STRAIGHT64, sb.VAR_WARP, sb.VAR_WARP64, 21, 22, 24, 28, 41, 42, 44, 48, 61, 62,
            64, 68, sb.VAR_COL[4], sb.VAR_COL[8], sb.VAR_COL_GROUPS,
            sb.VAR_COOP1, sb.VAR_GENERIC]
CLASSES = [(0, 0, 0, 0), (1, 0, 1, 0), (1, 1, 1, 1), (2, 1, 2, 0), (2, 2, 1, 1), (2, 2, 2, 2),
           (3, 1, 2, 1), (3, 2, 1, 0), (2, 3, 3, 0), (3, 3, 2, 2), (4, 2, 1, 1), (3, 3, 3, 3)]


@pytest.fixture(scope="module")
def libs():
    lib = sb.load()
    lib.simint_init()
    lib.simint_b200_set_ordering(0)
    return lib, load_oracle()


def _case(lib, orc, am, deriv, seed):
    rng = np.random.default_rng(seed)
    big = sum(am) >= 9
    shells, grp = class_shells(rng, am, nsh=(1, 1, 1, 1) if big else (2, 1, 2, 1),
                               nprim=(1, 2) if big else (1, 3))
    S = ShellSet(shells)
    orc.oracle_normalize_shells(S.n, S.ptr(0))
    bra = [(i, j) for i in grp[0] for j in grp[1]]
    ket = [(i, j) for i in grp[2] for j in grp[3]]
    oP, oQ = oracle_pairs(orc, S, bra), oracle_pairs(orc, S, ket)
    rr, ref = oracle_eri(orc, oP, oQ, 0.0, deriv, 0)
    orc.oracle_free_pair(C.byref(oP))
    orc.oracle_free_pair(C.byref(oQ))
    return S, bra, ket, rr, ref


@pytest.mark.parametrize("deriv", [0, 1])
@pytest.mark.parametrize("am", CLASSES, ids=lambda a: "".join("spdfg"[x] for x in a))
def test_every_variant_matches_oracle(libs, am, deriv):
    lib, orc = libs
    if deriv and sum(am) > 8:
        pytest.skip("deriv=1 sampled up to l_total 8 here")
    S, bra, ket, rr, ref = _case(lib, orc, am, deriv, 4242 + 13 * sum(am) + am[0] + deriv)
    P = sb.make_pairs(lib, S, bra)
    Q = sb.make_pairs(lib, S, ket)
    ran = []
    try:
        for v in VARIANTS:
            if sb.set_variant(am, v, deriv, sb.FP64, lib) != 0:
                continue
            ran.append(v)
            r, out = sb.compute_eri(P, Q, 0.0, deriv, lib)
            assert r == rr, (v, r, rr)
            bad, dmax = parity_bad(out, ref)
            assert len(bad) == 0, (v, dmax)
    finally:
        sb.set_variant(am, sb.VAR_DEFAULT, deriv, sb.FP64, lib)
        lib.simint_free_multi_shellpair(C.byref(P))
        lib.simint_free_multi_shellpair(C.byref(Q))
    assert sb.VAR_GENERIC in ran and len(ran) >= 2, ran


@pytest.mark.parametrize("am", [(2, 2, 2, 2), (3, 2, 2, 1)], ids=lambda a: "".join("spdfg"[x] for x in a))
def test_fp64_forms_under_mixed_mode(libs, am):
    """Codes 100 + v run the cooperative kernel without its FP32 path in
    mixed mode: FP64 parity holds whatever the gate."""
    lib, orc = libs
    S, bra, ket, rr, ref = _case(lib, orc, am, 0, 99 + sum(am))
    P = sb.make_pairs(lib, S, bra, sb.SIMINT_SCREEN_SCHWARZ)
    Q = sb.make_pairs(lib, S, ket, sb.SIMINT_SCREEN_SCHWARZ)
    try:
        lib.simint_b200_set_precision(sb.MIXED, 1e30)
        for v in (124, 142):
            assert sb.set_variant(am, v, 0, sb.MIXED, lib) == 0
            r, out = sb.compute_eri(P, Q, 0.0, 0, lib)
            bad, dmax = parity_bad(out, ref)
            assert len(bad) == 0, (v, dmax)
        assert sb.set_variant(am, 124, 0, sb.FP64, lib) != 0       # mixed mode only
    finally:
        lib.simint_b200_set_precision(sb.FP64, 0.0)
        sb.set_variant(am, sb.VAR_DEFAULT, 0, sb.MIXED, lib)
        lib.simint_free_multi_shellpair(C.byref(P))
        lib.simint_free_multi_shellpair(C.byref(Q))


@pytest.mark.parametrize("am", [(2, 1, 2, 1), (3, 2, 1, 0)], ids=["dpdp", "fdps"])
def test_fp32_batches_agree_across_cooperative_variants(libs, am):
    """Mixed mode with a loose gate sends most primitive quartets through the
    FP32 batches (2B of them, at most 8, per batch); every thread count and
    batch size must give the same integrals as batch 1 (the VRR of a
    primitive quartet does not depend on its batch, the sums run in
    primitive order)."""
    lib, orc = libs
    rng = np.random.default_rng(2718 + sum(am))
    shells, grp = class_shells(rng, am, nsh=(2, 1, 2, 1), nprim=(3, 4), alpha=(0.3, 30.0))
    S = ShellSet(shells)
    orc.oracle_normalize_shells(S.n, S.ptr(0))
    P = sb.make_pairs(lib, S, [(i, j) for i in grp[0] for j in grp[1]])
    Q = sb.make_pairs(lib, S, [(i, j) for i in grp[2] for j in grp[3]])
    outs = {}
    try:
        lib.simint_b200_set_precision(sb.MIXED, 1e-3)
        for v in (21, 22, 24, 28, 41, 42, 44, 48, 61, 62, 64, 68):
            if sb.set_variant(am, v, 0, sb.MIXED, lib) != 0:
                continue
            r, outs[v] = sb.compute_eri(P, Q, 0.0, 0, lib)
    finally:
        lib.simint_b200_set_precision(sb.FP64, 0.0)
        sb.set_variant(am, sb.VAR_DEFAULT, 0, sb.MIXED, lib)
        lib.simint_free_multi_shellpair(C.byref(P))
        lib.simint_free_multi_shellpair(C.byref(Q))
    assert 21 in outs and 28 in outs, sorted(outs)
    scale = float(np.abs(outs[21]).max())
    for v, o in outs.items():
        assert np.abs(o - outs[21]).max() <= 1e-13 * scale, (v, np.abs(o - outs[21]).max(), scale)
