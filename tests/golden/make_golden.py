"""Generate the golden fixtures of tests/golden from the reference itself.

Run here, where the reference tree is present:

    python oracle/build.py          # builds oracle/_ref/libsimint_ref.so
    python tests/golden/make_golden.py

The reference-built library is compiled from the reference's own sources
(oracle/build.py): its long-double test oracle ValeevRef
(skel/test/ValeevRef.cpp, the values the reference's test_eri and
test_eri_deriv1 compare against), its Boys function (skel/simint/boys) and
its pair code (skel/simint/shell/shell.c).  Inputs are seeded synthetic
shells normalised with the reference's simint_normalize_shells.

Outputs (numpy .npz, a few hundred kB in total):
  valeev_deriv0.npz  every class up to (dd|dd), Psi4 order
  valeev_deriv1.npz  every class up to (pp|pp) and a set of d classes
  valeev_fg.npz      f and g classes (deriv 0) with 1-3 primitives, exponents
                     in [0.05, 5e4] (the benchmark configurations' range; each
                     shell's first primitive diffuse, 0.05-5) and shells on two
                     pseudo-atoms in a 2 bohr box; ValeevRef in Psi4 order
  valeev_fg_d1.npz   f classes, deriv 1, the same ranges
  boys_ref.npz       reference boys_F_split values and grid rows
  pairs_ref.npz      reference multi-shell-pair arrays (no screening and
                     fast Schwarz), for bit-exact checks of our pair code
  oei_ref.npz        reference one-electron integrals (overlap, kinetic
                     energy, nuclear attraction; skel/simint/osoei) for every
                     (la|lb) up to (g|g)

`--oei-only` regenerates oei_ref.npz alone; `--fg-only` the f/g files alone.
"""

import ctypes as C
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "simint-generator_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from simint_b200.capi import ShellSet, ShellP, SimintMultiShellpair, pair_arrays  # noqa: E402
from simint_b200.workloads import random_shells  # noqa: E402
from oracle import load_ref  # noqa: E402

NC = lambda l: (l + 1) * (l + 2) // 2


def shells_to_arrays(shells):
    am = np.array([s[0] for s in shells], np.int32)
    xyz = np.array([s[1] for s in shells], float)
    nprim = np.array([len(s[2]) for s in shells], np.int32)
    alpha = np.concatenate([s[2] for s in shells])
    coef = np.concatenate([s[3] for s in shells])
    return dict(am=am, xyz=xyz, nprim=nprim, alpha=alpha, coef=coef)


def normalized(ref, shells):
    S = ShellSet(shells)
    ref.simint_normalize_shells(S.n, S.ptr(0))
    return S


def valeev(ref, S, grp, deriv):
    sub = [S.subset(g) for g in grp]
    n = 1
    for k in range(4):
        n *= len(grp[k]) * NC(S.arr[grp[k][0]].am)
    out = np.zeros(n * (12 if deriv else 1))
    ref.ref_valeev_integrals(C.cast(sub[0], ShellP), len(grp[0]), C.cast(sub[1], ShellP), len(grp[1]),
                             C.cast(sub[2], ShellP), len(grp[2]), C.cast(sub[3], ShellP), len(grp[3]),
                             out.ctypes.data_as(C.POINTER(C.c_double)), deriv)
    return out


def make_valeev(ref, deriv, classes, nsh, nprim, seed, alpha=(0.15, 12.0), box=2.5, shell_fn=None):
    rng = np.random.default_rng(seed)
    data = {}
    for am in classes:
        ams = sum(([am[k]] * nsh[k] for k in range(4)), [])
        if shell_fn:
            shells = shell_fn(rng, ams, nprim=nprim)
        else:
            shells = random_shells(rng, ams, nprim_range=nprim, alpha=alpha, box=box)
        S = normalized(ref, shells)
        # store the normalised coefficients so users skip normalisation
        norm = [(s[0], s[1], s[2], S.coefs(k)) for k, s in enumerate(shells)]
        idx = np.cumsum([0] + list(nsh))
        grp = [list(range(idx[k], idx[k + 1])) for k in range(4)]
        vals = valeev(ref, S, grp, deriv)
        key = "".join("spdfg"[x] for x in am)
        for k, v in shells_to_arrays(norm).items():
            data[key + "/" + k] = v
        data[key + "/nsh"] = np.array(nsh, np.int32)
        data[key + "/values"] = vals
        print(deriv, key, vals.size, flush=True)
    return data


def make_boys(ref):
    xs = np.concatenate([np.linspace(0, 40, 401), [1e-12, 0.049999, 0.05, 36.49, 36.5, 36.51, 50, 120]])
    F = np.zeros((len(xs), 17, 17))
    for a, x in enumerate(xs):
        for n in range(17):
            buf = np.zeros(32)
            ref.ref_boys_F(float(x), n, buf.ctypes.data_as(C.POINTER(C.c_double)))
            F[a, n, :n + 1] = buf[:n + 1]
    rows = np.array([[ref.ref_boys_grid(i, n) for n in range(32)] for i in range(366)])
    longfac = np.array([ref.ref_boys_longfac(n) for n in range(32)])
    return dict(x=xs, F=F, grid=rows, longfac=longfac)


def make_pairs(ref):
    rng = np.random.default_rng(4242)
    shells = random_shells(rng, [0, 1, 2, 1, 0, 2, 3, 1, 0, 1], nprim_range=(1, 5),
                           alpha=(0.1, 50.0), box=4.0)
    S = normalized(ref, shells)
    norm = [(s[0], s[1], s[2], S.coefs(k)) for k, s in enumerate(shells)]
    data = {"shells/" + k: v for k, v in shells_to_arrays(norm).items()}
    # pair lists: includes a shell with itself and > 16 pairs (padding)
    lists = {"mixed": [(i, j) for i in range(10) for j in range(10) if (i + j) % 3 == 0],
             "self": [(3, 3), (1, 1), (3, 1)]}
    for name, pl in lists.items():
        for screen in (0, 2):
            P = SimintMultiShellpair()
            ref.simint_initialize_multi_shellpair(C.byref(P))
            arr = S.pair_list(pl)
            ref.simint_create_multi_shellpair2(len(pl), C.cast(arr, ShellP), C.byref(P), screen)
            a = pair_arrays(P)
            pre = "%s_%d/" % (name, screen)
            data[pre + "pairs"] = np.array(pl, np.int32)
            for k, v in a.items():
                if v is None:
                    continue
                data[pre + k] = np.asarray(v)
            ref.simint_free_multi_shellpair(C.byref(P))
    return data


def make_oei(ref):
    """Reference one-electron integrals (skel/simint/osoei): overlap, kinetic
    energy and nuclear attraction of every (la, lb) up to (g|g), two shells
    per side (shared centres included), six point charges."""
    rng = np.random.default_rng(777)
    dp = C.POINTER(C.c_double)
    data = {}
    for la in range(5):
        for lb in range(5):
            shells = random_shells(rng, [la, la, lb, lb], nprim_range=(1, 4), alpha=(0.05, 5e3),
                                   box=3.0, natom=3)
            S = normalized(ref, shells)
            norm = [(s[0], s[1], s[2], S.coefs(k)) for k, s in enumerate(shells)]
            cen = rng.uniform(-1.0, 4.0, (6, 3))
            Z = rng.integers(1, 19, 6).astype(float)
            X, Y, Zc = (np.ascontiguousarray(cen[:, k]) for k in range(3))
            n = NC(la) * NC(lb)
            vals = np.zeros((3, 2, 2, n))
            for a in range(2):
                for b in range(2):
                    A, B = S.ptr(a), S.ptr(2 + b)
                    ref.simint_compute_osoei_overlap(A, B, vals[0, a, b].ctypes.data_as(dp))
                    ref.simint_compute_osoei_ke(A, B, vals[1, a, b].ctypes.data_as(dp))
                    ref.simint_compute_osoei_potential(6, Z.ctypes.data_as(dp), X.ctypes.data_as(dp),
                                                       Y.ctypes.data_as(dp), Zc.ctypes.data_as(dp),
                                                       A, B, vals[2, a, b].ctypes.data_as(dp))
            key = "spdfg"[la] + "spdfg"[lb]
            for k, v in shells_to_arrays(norm).items():
                data[key + "/" + k] = v
            data[key + "/centres"] = np.concatenate([cen, Z[:, None]], axis=1)
            data[key + "/values"] = vals
    return data


def main():
    ref = load_ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libsimint_ref.so missing: run python oracle/build.py here")
    if "--fg-only" in sys.argv:
        make_fg(ref)
        return
    np.savez_compressed(os.path.join(HERE, "oei_ref.npz"), **make_oei(ref))
    if "--oei-only" in sys.argv:
        return
    d0 = list(itertools.product(range(3), repeat=4))
    np.savez_compressed(os.path.join(HERE, "valeev_deriv0.npz"),
                        **make_valeev(ref, 0, d0, (1, 2, 1, 1), (1, 2), 11))
    d1 = list(itertools.product(range(2), repeat=4)) + [(2, 0, 0, 0), (0, 0, 2, 1), (2, 1, 1, 0),
                                                         (1, 2, 0, 1), (2, 2, 1, 1), (2, 0, 2, 0)]
    # ValeevRef's deriv=1 output is only laid out correctly for one shell in
    # the first position (its offset omits the factor 12), so nsh[0] = 1
    np.savez_compressed(os.path.join(HERE, "valeev_deriv1.npz"),
                        **make_valeev(ref, 1, d1, (1, 1, 2, 1), (1, 2), 12))
    np.savez_compressed(os.path.join(HERE, "boys_ref.npz"), **make_boys(ref))
    np.savez_compressed(os.path.join(HERE, "pairs_ref.npz"), **make_pairs(ref))
    make_fg(ref)


# f and g classes of the benchmark workloads (the dominant (fd|fp), (fd|dp),
# (ff|fd) of the l <= 3 sweep, g classes of the l <= 4 sweep)
FG_D0 = [(3, 0, 0, 0), (3, 0, 3, 0), (3, 1, 3, 0), (3, 2, 1, 1), (3, 2, 2, 1), (3, 2, 3, 1),
         (3, 3, 2, 2), (3, 3, 3, 2), (3, 3, 3, 3), (2, 2, 3, 3), (4, 0, 0, 0), (4, 1, 2, 0),
         (4, 0, 4, 0), (4, 2, 3, 1), (4, 4, 0, 0), (4, 3, 2, 2), (4, 4, 2, 1)]
FG_D1 = [(3, 0, 0, 0), (3, 1, 1, 0), (3, 2, 1, 1), (3, 1, 2, 2), (2, 2, 3, 0)]


def fg_shells(rng, ams, nprim=(1, 3), alpha=(0.05, 5e4), box=2.0, natom=2):
    """Shells for the f/g fixtures: exponents log-uniform over the
    configurations' range, except that every shell's first primitive is
    diffuse (0.05-5), as in contracted shells, so that quartets across the
    two pseudo-atoms do not all underflow."""
    atoms = rng.uniform(0.0, box, size=(natom, 3))
    out = []
    for k, am in enumerate(ams):
        n = int(rng.integers(nprim[0], nprim[1] + 1))
        al = np.exp(rng.uniform(np.log(alpha[0]), np.log(alpha[1]), size=n))
        al[0] = np.exp(rng.uniform(np.log(0.05), np.log(5.0)))
        co = rng.uniform(0.1, 1.0, size=n)
        out.append((int(am), tuple(atoms[k % natom]), al, co))
    return out


def _fg_one(job):
    """One f/g class in a worker process (its own reference library handle
    and a seed of its own, so the result does not depend on the order)."""
    deriv, am, nsh, nprim, seed = job
    ref = load_ref()
    return make_valeev(ref, deriv, [am], nsh, nprim, seed, shell_fn=fg_shells)


def make_fg(ref, workers=None):
    """valeev_fg.npz / valeev_fg_d1.npz: one class per process (ValeevRef in
    long double takes minutes for the largest of them)."""
    import multiprocessing as mp
    jobs0 = [(0, am, (1, 1, 1, 1), (1, 3), 1300 + k) for k, am in enumerate(FG_D0)]
    jobs1 = [(1, am, (1, 1, 1, 1), (1, 3), 1400 + k) for k, am in enumerate(FG_D1)]
    with mp.get_context("fork").Pool(workers or os.cpu_count()) as pool:
        res = pool.map(_fg_one, jobs0 + jobs1, chunksize=1)
    d0, d1 = {}, {}
    for job, r in zip(jobs0 + jobs1, res):
        (d1 if job[0] else d0).update(r)
    for name, d in (("valeev_fg.npz", d0), ("valeev_fg_d1.npz", d1)):
        tmp = os.path.join(HERE, "." + name + ".tmp.npz")
        np.savez_compressed(tmp, **d)
        os.replace(tmp, os.path.join(HERE, name))


if __name__ == "__main__":
    main()
