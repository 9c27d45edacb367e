"""GPU: simint_compute_eri from several host threads at once (each thread
has its own stream and device buffers in the library, as an OpenMP loop over
bra pairs calls the reference): every call's integrals equal the same call
made alone, bit for bit, for register-kernel and cooperative-kernel classes
and for a pipelined call ((ff|dd), 26 MB of results); concurrent first calls
of a fresh process initialise the library's tables once."""
import ctypes as C
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [((0, 0), (0, 0), 60), ((1, 0), (1, 1), 80), ((2, 1), (2, 0), 40), ((3, 2), (2, 1), 30),
         ((3, 3), (3, 1), 12), ((3, 3), (2, 2), 900)]


def _calls(lib):
    rng = np.random.default_rng(404)
    ams = [0] * 30 + [1] * 30 + [2] * 30 + [3] * 12
    shells = random_shells(rng, ams, nprim_range=(1, 4), alpha=(0.1, 50.0), box=6.0, natom=8)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    by = {l: [i for i, a in enumerate(ams) if a == l] for l in range(4)}
    calls = []
    for (a, b), (c, d), nk in CASES:
        P = sb.make_pairs(lib, S, [(by[a][0], by[b][1])], sb.SIMINT_SCREEN_SCHWARZ)
        kets = [(i, j) for i in by[c] for j in by[d]][:nk]
        Q = sb.make_pairs(lib, S, kets, sb.SIMINT_SCREEN_SCHWARZ)
        calls.append((P, Q))
    return S, calls


def test_concurrent_calls_equal_single_calls():
    lib = sb.load()
    lib.simint_init()
    S, calls = _calls(lib)
    try:
        alone = [sb.compute_eri(P, Q, 1e-14, 0, lib) for P, Q in calls]
        work = [k for k in range(len(calls)) for _ in range(4)]
        with ThreadPoolExecutor(max_workers=8) as pool:
            got = list(pool.map(lambda k: (k, sb.compute_eri(calls[k][0], calls[k][1], 1e-14, 0, lib)), work))
        for k, (r, out) in got:
            assert r == alone[k][0]
            assert np.array_equal(out, alone[k][1]), CASES[k]
    finally:
        for P, Q in calls:
            lib.simint_free_multi_shellpair(C.byref(P))
            lib.simint_free_multi_shellpair(C.byref(Q))


CHILD = r"""
import numpy as np, ctypes as C
from concurrent.futures import ThreadPoolExecutor
import simint_b200 as sb
import test_gpu_threads as t
lib = sb.load(); lib.simint_init()
S, calls = t._calls(lib)
with ThreadPoolExecutor(max_workers=6) as pool:
    got = list(pool.map(lambda k: sb.compute_eri(calls[k][0], calls[k][1], 1e-14, 0, lib), range(len(calls))))
alone = [sb.compute_eri(P, Q, 1e-14, 0, lib) for P, Q in calls]
print(all(g[0] == a[0] and np.array_equal(g[1], a[1]) for g, a in zip(got, alone)))
"""


def test_concurrent_first_calls():
    """The first calls of a process come from six threads at once."""
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([os.path.join(ROOT, "simint-generator_b200"), os.path.join(ROOT, "tests"),
                                         env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().endswith("True"), r.stdout[-500:]
