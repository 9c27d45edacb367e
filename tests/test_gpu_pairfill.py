"""GPU: the Gaussian-product fill of simint_create_multi_shellpair2 on the
device (simint_b200_set_pair_fill) against the host fill, which equals the
reference's shell.c bit for bit (tests/test_oracle_pins.py).

Per shell pair the GPU fill must give the same primitive pairs: centres,
P - A, P - B, exponent sums, 2a and 2b, A - B and counts bit for bit, the
prefactors within a few ulps (CUDA's exp against the host's), the screening
values keeping and dropping the same primitive pairs at every threshold from
1e-16 to 1e-32 (their (ab|ab) evaluations round differently on inputs a few
ulps apart, so values far below a pair's largest carry relative noise), in
decreasing screening order; the
padding slots bit for bit.  A pair of a shell with itself keeps the i >= j
triangle with doubled off-diagonal prefactors.  The integrals from the two
fills agree to 1e-12 of their largest magnitude without screening and 1e-9
with it (primitive order within rounding ties), below (ff|ff), whose
conditioning on these shells (exponents 0.05-5e4) exceeds that."""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet, pair_arrays, padded_nprim
from simint_b200.workloads import random_shells

pytestmark = pytest.mark.gpu

EXACT = ("x", "y", "z", "PA_x", "PA_y", "PA_z", "PB_x", "PB_y", "PB_z", "alpha", "alpha2", "beta2")


def _pairs(lib, S, pairs, screen, mode):
    assert sb.set_pair_fill(mode, lib) == 0
    try:
        n0 = lib.simint_b200_launch_count()
        P = sb.make_pairs(lib, S, pairs, screen)
        return P, lib.simint_b200_launch_count() - n0
    finally:
        sb.set_pair_fill(sb.PAIR_FILL_AUTO, lib)


def _starts(a):
    st, idx = [], 0
    n = a["nshell12"]
    for p in range(n):
        st.append(idx)
        idx += int(a["nprim12"][p])
        if (p + 1) % 16 == 0 or p + 1 >= n:
            idx = (idx + 7) & ~7
    return st, idx


def _compare(h, g, screen):
    for k in ("am1", "am2", "nprim", "nshell12", "nshell12_clip", "screen_max"):
        assert h[k] == g[k], k
    for k in ("nprim12", "AB_x", "AB_y", "AB_z"):
        assert np.array_equal(h[k], g[k]), k
    st, npad = _starts(h)
    used = np.zeros(npad, bool)
    for p, s0 in enumerate(st):
        n = int(h["nprim12"][p])
        sl = slice(s0, s0 + n)
        used[sl] = True
        # the same primitive pairs, in the order of each fill's screening
        # values (ties within rounding may come out in either order)
        key = lambda a: np.lexsort((a["z"][sl], a["y"][sl], a["x"][sl], a["alpha2"][sl], a["alpha"][sl]))
        oh, og = key(h), key(g)
        for k in EXACT:
            assert np.array_equal(h[k][sl][oh], g[k][sl][og]), (k, p)
        ph, pg = h["prefac"][sl][oh], g["prefac"][sl][og]
        assert np.all(np.abs(ph - pg) <= 4 * np.spacing(np.abs(ph))), p
        if screen:
            sh, sg = h["screen"][sl][oh], g["screen"][sl][og]
            # (ab|ab) of a primitive pair from prefactors a few ulps apart:
            # the rounding of its recurrences differs, and the rounding error
            # of a value scales with the largest intermediates, so values far
            # below them carry relative noise (a 5.1e-21 value beside a
            # 5.9e-3 one moved by 3e-7 of itself).  A screening value is only
            # compared with tol^2: the two fills must keep and drop the same
            # primitive pairs at every threshold, except values within 1e-3
            # of it, and agree to 1e-3 of the pair's scale (gross errors).
            scale = float(np.abs(sh).max())
            assert np.all(np.abs(sh - sg) <= 1e-3 * np.abs(sh) + 1e-6 * scale + 1e-40), p
            for t in (1e-16, 1e-20, 1e-24, 1e-28, 1e-32):
                near = np.abs(sh - t) <= 1e-3 * t
                assert np.array_equal((sh >= t) | near, (sg >= t) | near), (p, t)
            assert np.all(np.diff(g["screen"][sl]) <= 0.0), p
            # where the host order has no near-ties the orders agree
            d = np.diff(h["screen"][sl])
            if n > 1 and np.all(-d > 1e-5 * np.abs(h["screen"][sl][1:]) + 1e-9 * float(np.abs(sh).max())):
                for k in EXACT:
                    assert np.array_equal(h[k][sl], g[k][sl]), (k, p)
    for k in EXACT + ("prefac",) + (("screen",) if screen else ()):
        assert np.array_equal(h[k][~used], g[k][~used]), k


@pytest.mark.parametrize("screen", [sb.SIMINT_SCREEN_NONE, sb.SIMINT_SCREEN_SCHWARZ,
                                    sb.SIMINT_SCREEN_FASTSCHWARZ])
@pytest.mark.parametrize("am", [(0, 0), (2, 1), (2, 2), (3, 3)])
def test_gpu_fill_equals_host_fill(am, screen):
    lib = sb.load()
    lib.simint_init()
    rng = np.random.default_rng(101 + 7 * am[0] + am[1] + 13 * screen)
    na, nb = 9, 7
    shells = random_shells(rng, [am[0]] * na + [am[1]] * nb, nprim_range=(1, 6), alpha=(0.05, 5e4),
                           box=6.0, natom=5)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    pairs = [(i, j) for i in range(na) for j in range(na, na + nb)]
    if am[0] == am[1]:
        # shells with themselves (i >= j triangles) and repeated pairs
        pairs += [(i, i) for i in range(na)] + [(j, i) for i in range(na) for j in range(i)]
    Ph, _ = _pairs(lib, S, pairs, screen, sb.PAIR_FILL_HOST)
    Pg, nl = _pairs(lib, S, pairs, screen, sb.PAIR_FILL_GPU)
    try:
        assert nl >= 1
        _compare(pair_arrays(Ph), pair_arrays(Pg), screen)
        # integrals from the two fills
        Q = [(i, j) for i in range(na) for j in range(na, na + nb)][:24]
        Qh, _ = _pairs(lib, S, Q, screen, sb.PAIR_FILL_HOST)
        Qg, _ = _pairs(lib, S, Q, screen, sb.PAIR_FILL_GPU)
        Ph.nshell12_clip = Pg.nshell12_clip = min(Ph.nshell12, 40)
        r1, o1 = sb.compute_eri(Ph, Qh, 1e-14 if screen else 0.0, 0, lib)
        r2, o2 = sb.compute_eri(Pg, Qg, 1e-14 if screen else 0.0, 0, lib)
        assert r1 == r2
        # prefactors a few ulps apart, amplified by the cancellation of the
        # tight (5e4) and diffuse (0.05) primitives of this set; (ff|ff) of
        # such shells is conditioned so that ulp changes of the inputs move
        # integrals by up to 1e-6 of their magnitude (the reference library
        # and the double oracle miss the long-double values by as much), so
        # the integrals are compared below it
        # with screening the two fills may order a shell pair's primitives
        # differently where screening values are within rounding of each
        # other, so the contraction sums in another order: 1e-9 there
        if r1 > 0 and am != (3, 3):
            bar = 1e-9 if screen else 1e-12
            assert np.abs(o1 - o2).max() <= bar * max(1.0, float(np.abs(o1).max()))
        Ph.nshell12_clip = Ph.nshell12
        Pg.nshell12_clip = Pg.nshell12
        lib.simint_free_multi_shellpair(C.byref(Qh))
        lib.simint_free_multi_shellpair(C.byref(Qg))
    finally:
        lib.simint_free_multi_shellpair(C.byref(Ph))
        lib.simint_free_multi_shellpair(C.byref(Pg))


def test_auto_mode_uses_gpu_for_large_lists():
    """Automatic mode: lists of 4096 or more padded primitive pairs on the
    GPU (one launch without screening), smaller ones on the host (none)."""
    lib = sb.load()
    lib.simint_init()
    rng = np.random.default_rng(77)
    shells = random_shells(rng, [1] * 40, nprim_range=(4, 6), alpha=(0.1, 100.0), box=8.0)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    big = [(i, j) for i in range(40) for j in range(40)]
    small = big[:20]
    assert sb.get_pair_fill(lib) == sb.PAIR_FILL_AUTO
    Pb, nb = _pairs(lib, S, big, sb.SIMINT_SCREEN_NONE, sb.PAIR_FILL_AUTO)
    Ps, ns = _pairs(lib, S, small, sb.SIMINT_SCREEN_NONE, sb.PAIR_FILL_AUTO)
    try:
        assert padded_nprim(Pb) >= 4096 and padded_nprim(Ps) < 4096
        assert nb == 1 and ns == 0
        Ph, _ = _pairs(lib, S, big, sb.SIMINT_SCREEN_NONE, sb.PAIR_FILL_HOST)
        _compare(pair_arrays(Ph), pair_arrays(Pb), False)
        lib.simint_free_multi_shellpair(C.byref(Ph))
    finally:
        lib.simint_free_multi_shellpair(C.byref(Pb))
        lib.simint_free_multi_shellpair(C.byref(Ps))
