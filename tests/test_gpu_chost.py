"""GPU: the reference's own C and C++ callers, compiled unchanged against
include/ and linked to libsimint_b200.so (oracle/build_chost.py).

* skel/examples/example1.c (water/STO-3G, every class up to (pp|pp)): its
  output must equal the output of the same program linked to the reference's
  generated library.
* skel/test/test_eri.cpp with the reference's long-double ValeevRef: every
  AM class of water in the 6-31G** and DZP basis sets must pass the
  reference's own acceptance rule (test_eri.cpp:227; a failing class is
  printed with "***").
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def need(name):
    p = os.path.join(REF, name)
    if not os.path.exists(p):
        pytest.skip("%s not built (oracle/build_chost.py)" % name)
    return p


def test_example1_matches_reference_build():
    exe = need("example1_b200")
    want = open(need("example1_ref.out")).read()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout == want


@pytest.mark.parametrize("mol,nclass", [("water.6-31gss.mol", 81), ("water.dzp.mol", 81)])
def test_test_eri_against_valeev(mol, nclass):
    exe = need("test_eri_b200")
    basis = need(os.path.join("dat", mol))
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run([exe, basis], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("(")]
    assert len(lines) == nclass, r.stdout[-2000:]
    bad = [l for l in lines if "***" in l]
    assert not bad, bad
