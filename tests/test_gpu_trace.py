"""GPU: the opt-in call trace (SIMINT_B200_TRACE=1) prints one phase line per
simint_compute_eri call on stderr and does not change the results; without
the variable nothing is printed.  Runs in child processes, since the library
reads the variable once."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHILD = r"""
import numpy as np, simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells
lib = sb.load(); lib.simint_init()
S = ShellSet(random_shells(np.random.default_rng(3), [2, 1, 1, 0], nprim_range=(1, 3), box=3.0))
lib.simint_normalize_shells(S.n, S.ptr(0))
P = sb.make_pairs(lib, S, [(0, 1)]); Q = sb.make_pairs(lib, S, [(2, 3)])
r, out = sb.compute_eri(P, Q, 0.0, 0, lib)
print(r, repr(float(np.abs(out).sum())))
"""


def _run(trace):
    env = dict(os.environ)
    env["PYTHONPATH"] = os.path.join(ROOT, "simint-generator_b200") + os.pathsep + env.get("PYTHONPATH", "")
    env.pop("SIMINT_B200_TRACE", None)
    if trace:
        env["SIMINT_B200_TRACE"] = "1"
    return subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)


def test_trace_lines_and_unchanged_results():
    plain, traced = _run(False), _run(True)
    assert plain.returncode == 0 and traced.returncode == 0, (plain.stderr, traced.stderr)
    assert plain.stdout == traced.stdout
    assert "simint_b200 trace" not in plain.stderr
    lines = [l for l in traced.stderr.splitlines() if l.startswith("simint_b200 trace:")]
    assert len(lines) == 1
    assert "(2 1|1 0)" in lines[0] and "pack" in lines[0] and "wait" in lines[0] and "copy" in lines[0]
