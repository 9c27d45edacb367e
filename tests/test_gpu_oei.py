"""GPU: one-electron integrals (overlap, kinetic energy, nuclear attraction).

* the reference's per-pair calls (simint_compute_overlap / _ke / _potential)
  against golden values made by the reference's own osoei code
  (tests/golden/oei_ref.npz, every (la|lb) up to (g|g)), and against the CPU
  oracle on wide-exponent random shells in both shell orders;
* the batched matrices (simint_b200_oei_matrix) against blocks assembled from
  the oracle, in both Cartesian orderings;
* edge cases: no centres, a shell with itself, far-apart shells, am 5.

Bar per block: |d| <= 1e-13 * max(1, max |block|) (values reach 1e3-1e4 for
tight exponents), or, where the evaluation cancels (the kinetic energy's
a - 2a^2 (PA^2 + 1/2p) at tight exponents), the GPU is at least as close to
the long-double evaluation of the same formulas as the double-precision
reference or oracle is (within twice its largest error plus 1e-15 of the
block scale).  The GPU's nuclear attraction uses the bra-side recursion plus
a horizontal transfer and contracts a*b+c into FMAs; the reference recurses
on both centres, so the two round differently."""
import os

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells
from oracle import load_oracle, load_oracle_ld
from _util import oracle_oei, NC

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
OEI = np.load(os.path.join(GOLD, "oei_ref.npz"))
TOL = 1e-13


def _shells(key):
    am, xyz, nprim = OEI[key + "/am"], OEI[key + "/xyz"], OEI[key + "/nprim"]
    al, co = OEI[key + "/alpha"], OEI[key + "/coef"]
    out, o = [], 0
    for s in range(len(am)):
        n = int(nprim[s])
        out.append((int(am[s]), tuple(xyz[s]), al[o:o + n], co[o:o + n]))
        o += n
    return out


_LD = []


def _ld():
    if not _LD:
        _LD.append(load_oracle_ld())
    return _LD[0]


def _close(calc, ref, tol=TOL, exact=None):
    """calc within tol of ref (block scale), or -- given exact, the
    long-double values -- no further from exact than ref is (x2 + 1e-15)."""
    scale = max(1.0, float(np.abs(ref).max()) if ref.size else 1.0)
    d = float(np.abs(calc - ref).max()) if ref.size else 0.0
    if d <= tol * scale:
        return True, d, scale
    if exact is not None:
        e_ref = float(np.abs(ref - exact).max())
        e_calc = float(np.abs(calc - exact).max())
        return e_calc <= 2.0 * e_ref + 1e-15 * scale, d, scale
    return False, d, scale


@pytest.fixture(scope="module")
def lib():
    L = sb.load()
    L.simint_init()
    L.simint_b200_set_ordering(0)
    return L


@pytest.mark.parametrize("key", sorted({k.split("/")[0] for k in OEI.files}))
def test_pairs_match_reference_osoei(lib, key):
    S = ShellSet(_shells(key))
    cen = OEI[key + "/centres"]
    ref = OEI[key + "/values"]
    for kind in range(3):
        for a in range(2):
            for b in range(2):
                r, out = sb.compute_oei(kind, S, a, 2 + b, cen, lib)
                assert r == 1
                ok, d, scale = _close(out, ref[kind, a, b],
                                      exact=oracle_oei(_ld(), kind, S, a, 2 + b, cen))
                assert ok, (key, kind, a, b, d, scale)


def test_pairs_match_oracle_both_orders(lib):
    """Wide exponents (0.02-1e5), shared and distinct centres, both shell
    orders (the transposed classes are computed as the transpose)."""
    orc = load_oracle()
    rng = np.random.default_rng(901)
    worst = 0.0
    for la in range(5):
        for lb in range(5):
            shells = random_shells(rng, [la, lb], nprim_range=(1, 6), alpha=(0.02, 1e5), box=5.0, natom=2)
            S = ShellSet(shells)
            lib.simint_normalize_shells(S.n, S.ptr(0))
            cen = np.concatenate([rng.uniform(-1, 6, (7, 3)), rng.integers(1, 30, (7, 1))], axis=1)
            for kind in range(3):
                for a, b in ((0, 1), (1, 0)):
                    r, out = sb.compute_oei(kind, S, a, b, cen, lib)
                    exp = oracle_oei(orc, kind, S, a, b, cen)
                    ok, d, scale = _close(out, exp, exact=oracle_oei(_ld(), kind, S, a, b, cen))
                    worst = max(worst, d / scale)
                    assert ok, (la, lb, kind, a, b, d, scale)
    print("largest deviation / block scale:", worst)


@pytest.mark.parametrize("ordering", [0, 1])
def test_matrices_match_oracle(lib, ordering):
    torch = pytest.importorskip("torch")
    orc = load_oracle()
    rng = np.random.default_rng(314 + ordering)
    ams = [0, 1, 2, 3, 4, 2, 1, 0, 3, 2]
    shells = random_shells(rng, ams, nprim_range=(1, 5), alpha=(0.05, 5e3), box=5.0, natom=4)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    cen = np.concatenate([rng.uniform(0, 5, (6, 3)), rng.integers(1, 20, (6, 1))], axis=1)
    off = np.cumsum([0] + [NC(a) for a in ams])
    nbf = int(off[-1])
    # position of each lexicographic Cartesian in the chosen ordering
    gam = {2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
           3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2),
               (0, 1, 2), (1, 1, 1)]}

    def lex(l):
        return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]

    def pos(l):
        if ordering == 1 and l in gam:
            return [gam[l].index(c) for c in lex(l)]
        return list(range(NC(l)))

    lib.simint_b200_set_ordering(ordering)
    try:
        for kind in range(3):
            exp = np.zeros((nbf, nbf))
            ext = np.zeros((nbf, nbf))
            for a in range(S.n):
                for b in range(S.n):
                    blk = oracle_oei(orc, kind, S, a, b, cen).reshape(NC(ams[a]), NC(ams[b]))
                    bld = oracle_oei(_ld(), kind, S, a, b, cen).reshape(NC(ams[a]), NC(ams[b]))
                    pa, pb = pos(ams[a]), pos(ams[b])
                    for u in range(NC(ams[a])):
                        for v in range(NC(ams[b])):
                            exp[off[a] + pa[u], off[b] + pb[v]] = blk[u, v]
                            ext[off[a] + pa[u], off[b] + pb[v]] = bld[u, v]
            M = torch.full((nbf, nbf), float("nan"), dtype=torch.float64, device="cuda")
            sb.oei_matrix(kind, S, cen, M.data_ptr(), torch.cuda.current_stream().cuda_stream, lib)
            torch.cuda.synchronize()
            got = M.cpu().numpy()
            assert np.isfinite(got).all()          # every element written
            assert np.array_equal(got, got.T)
            for a in range(S.n):
                for b in range(S.n):
                    sl = (slice(off[a], off[a + 1]), slice(off[b], off[b + 1]))
                    ok, d, scale = _close(got[sl], exp[sl], exact=ext[sl])
                    assert ok, (kind, a, b, d, scale)
    finally:
        lib.simint_b200_set_ordering(0)


def test_edge_cases(lib):
    orc = load_oracle()
    rng = np.random.default_rng(5)
    shells = random_shells(rng, [2, 3], nprim_range=(2, 4), alpha=(0.1, 50.0), box=2.0, natom=2)
    far = (1, (500.0, 0.0, 0.0), [0.7, 2.0], [0.5, 0.5])
    S = ShellSet(shells + [far])
    lib.simint_normalize_shells(S.n, S.ptr(0))
    # no centres: the potential block is zero
    r, out = sb.compute_oei(2, S, 0, 1, np.zeros((0, 4)), lib)
    assert r == 1 and np.all(out == 0.0)
    # a shell with itself (A == B, same primitives)
    for kind in range(3):
        cen = [[0.3, 0.1, -0.2, 8.0]]
        r, out = sb.compute_oei(kind, S, 1, 1, cen, lib)
        ok, d, scale = _close(out, oracle_oei(orc, kind, S, 1, 1, cen),
                              exact=oracle_oei(_ld(), kind, S, 1, 1, cen))
        assert r == 1 and ok, (kind, d)
    # far apart: overlap and kinetic energy underflow to exact zeros, like the oracle
    for kind in range(2):
        r, out = sb.compute_oei(kind, S, 0, 2, None, lib)
        assert r == 1 and np.array_equal(out, oracle_oei(orc, kind, S, 0, 2))
    # am 5 is not built: a clean error, nothing written
    g = ShellSet([(5, (0.0, 0.0, 0.0), [1.0], [1.0]), (0, (0.0, 0.0, 1.0), [1.0], [1.0])])
    r, out = sb.compute_oei(0, g, 0, 1, None, lib)
    assert r == -3          # SIMINT_B200_ERR_CLASS
