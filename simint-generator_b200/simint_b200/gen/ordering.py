"""Cartesian orderings of Gaussian shells (Psi4 and GAMESS).

The ordering of the Cartesian components inside a shell of angular momentum l
decides where each integral lands in the output array.

* Psi4 order: lexicographically descending in the x exponent, then the y
  exponent.  It is produced by the iteration rule in
  python/ordering_common/ordering_psi4.py:3-13 (and its C++ twin
  IterateGaussian, skel/test/Common.cpp:20-33).
* GAMESS order (generator/Ordering_GAMESS.cpp:8-41) differs from Psi4 only at
  l = 2 and l = 3; for l = 0, 1 and l >= 4 the two tables are identical.

Both orderings are data of the interface (they decide the output layout), so
the l = 2 and l = 3 GAMESS lists below have to match the reference's tables.
"""

from functools import lru_cache

PSI4 = 0
GAMESS = 1
ORDERINGS = {"psi4": PSI4, "gamess": GAMESS}


def ncart(l):
    """Number of Cartesian components of a shell with angular momentum l."""
    return (l + 1) * (l + 2) // 2 if l >= 0 else 0


@lru_cache(maxsize=None)
def psi4_order(l):
    """Cartesian exponents (i, j, k) of a shell of AM l in Psi4 order."""
    out = []
    g = (l, 0, 0)
    while True:
        out.append(g)
        i, j, k = g
        if k == l:
            break
        if k < l - i:
            g = (i, j - 1, k + 1)
        else:
            g = (i - 1, l - i + 1, 0)
    return tuple(out)


_GAMESS_SPECIAL = {
    2: ((2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)),
    3: ((3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (2, 0, 1),
        (1, 2, 0), (0, 2, 1), (1, 0, 2), (0, 1, 2), (1, 1, 1)),
}


@lru_cache(maxsize=None)
def gamess_order(l):
    """Cartesian exponents of a shell of AM l in GAMESS order."""
    return _GAMESS_SPECIAL.get(l, psi4_order(l))


def order(l, ordering):
    return psi4_order(l) if ordering == PSI4 else gamess_order(l)


@lru_cache(maxsize=None)
def index_map(l, ordering):
    """dict (i, j, k) -> position of that Cartesian inside a shell of AM l."""
    return {g: n for n, g in enumerate(order(l, ordering))}


def cart_index(g, ordering):
    """Position of Cartesian exponent triple g inside its shell."""
    return index_map(sum(g), ordering)[g]


def psi4_to_gamess_perm(l):
    """perm[n] = GAMESS position of the n-th Psi4 Cartesian of AM l."""
    gm = index_map(l, GAMESS)
    return [gm[g] for g in psi4_order(l)]
