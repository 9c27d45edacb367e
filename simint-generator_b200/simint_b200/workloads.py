"""Seeded synthetic shell sets for the benchmark configurations.

Every configuration draws from numpy's PCG64 generator with seed 2024
(exponents log-uniform, contraction coefficients uniform in [0.1, 1], shells
normalised by simint_normalize_shells).  Shells of a configuration are
placed on pseudo-atoms: the shell list is shuffled and shell k goes to atom
k mod natom ("round robin after shuffling"); atoms are uniform in a cube.

  cfg1  64 shells (32 s, 32 p), 3 primitives, alpha in [0.1, 100],
        every shell on its own centre in an 8 bohr cube.
  cfg2  500 shells s:p:d:f = 200:150:100:50, 1-8 primitives,
        alpha in [0.05, 5e4], 120 atoms in a 20 bohr cube.
  cfg4  300 shells s:p:d = 150:100:50, 1-6 primitives, alpha in [0.1, 1e4],
        80 atoms in a 16 bohr cube.
  cfg5  2000 shells s:p:d:f:g = 667:533:400:267:133; primitives s,p 4-12,
        d 2-6, f,g 1-3; alpha in [0.02, 1e5]; 400 atoms in a 40 bohr cube.
"""

import numpy as np

SEED = 2024


def _shells(rng, counts, nprim_rule, alo, ahi, natom, box, own_centre=False):
    ams = []
    for am, n in enumerate(counts):
        ams += [am] * n
    ams = np.array(ams)
    order = rng.permutation(len(ams))
    ams = ams[order]
    if own_centre:
        centres = rng.uniform(0.0, box, size=(len(ams), 3))
    else:
        atoms = rng.uniform(0.0, box, size=(natom, 3))
        centres = atoms[np.arange(len(ams)) % natom]
    shells = []
    for k, am in enumerate(ams):
        nprim = int(nprim_rule(rng, int(am)))
        al = np.exp(rng.uniform(np.log(alo), np.log(ahi), size=nprim))
        co = rng.uniform(0.1, 1.0, size=nprim)
        shells.append((int(am), tuple(centres[k]), al, co))
    return shells


def config_shells(name, seed=SEED):
    rng = np.random.Generator(np.random.PCG64(seed))
    if name == "cfg1" or name == "cfg3":
        return _shells(rng, [32, 32], lambda r, am: 3, 0.1, 100.0, 0, 8.0, own_centre=True)
    if name == "cfg2":
        return _shells(rng, [200, 150, 100, 50], lambda r, am: r.integers(1, 9),
                       0.05, 5e4, 120, 20.0)
    if name == "cfg4":
        return _shells(rng, [150, 100, 50], lambda r, am: r.integers(1, 7),
                       0.1, 1e4, 80, 16.0)
    if name == "cfg5":
        def rule(r, am):
            if am <= 1:
                return r.integers(4, 13)
            if am == 2:
                return r.integers(2, 7)
            return r.integers(1, 4)
        return _shells(rng, [667, 533, 400, 267, 133], rule, 0.02, 1e5, 400, 40.0)
    raise KeyError(name)


def random_shells(rng, ams, nprim_range=(1, 4), alpha=(0.1, 20.0), box=3.0, natom=None):
    """Small random shell sets for parity tests."""
    shells = []
    if natom:
        atoms = rng.uniform(0.0, box, size=(natom, 3))
    for k, am in enumerate(ams):
        nprim = int(rng.integers(nprim_range[0], nprim_range[1] + 1))
        al = np.exp(rng.uniform(np.log(alpha[0]), np.log(alpha[1]), size=nprim))
        co = rng.uniform(0.1, 1.0, size=nprim)
        xyz = atoms[k % natom] if natom else rng.uniform(0.0, box, size=3)
        shells.append((int(am), tuple(xyz), al, co))
    return shells
