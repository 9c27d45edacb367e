"""Recipe: C and C++ hosts that drive libsimint_b200.so through its C ABI.

TEST INFRASTRUCTURE ONLY.  Everything is written to oracle/_ref/ (git-ignored;
it travels with the built library).

* oracle/_ref/librefdrv_b200.so -- oracle/refdrv.c (our driver of the public
  simint_* API) compiled against include/ and linked to libsimint_b200.so:
  the same C code that drives the reference's generated library in the
  oracle/_ref/libsimint_<variant>_<isa>.so builds, so a test can hand both
  libraries identical calls.
* oracle/_ref/example1_b200 -- the reference's skel/examples/example1.c
  compiled unchanged against include/, linked to libsimint_b200.so;
  oracle/_ref/example1_ref.out is the stdout of the same file built against
  the reference's generated library (gamess_l3), captured here.
* oracle/_ref/test_eri_b200 -- the reference's own accuracy test
  (skel/test/test_eri.cpp + Common.cpp + ValeevRef.cpp, its long-double
  oracle) compiled unchanged against include/ and linked to
  libsimint_b200.so; its acceptance rule (test_eri.cpp:227: a class fails
  when max abs error > 1e-14 and max rel error > 1e-8) marks failures with
  "***".  The basis files it reads are copied from skel/test/dat/ to
  oracle/_ref/dat/.

Usage: python oracle/build_chost.py [--ref PATH]  (reference tree from --ref
or $SIMINT_REFERENCE; without it only librefdrv_b200.so is built).
"""

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
INC = os.path.join(REPO, "include")
LIBDIR = os.path.join(REPO, "simint-generator_b200")
LIB = os.path.join(LIBDIR, "libsimint_b200.so")
MOLS = ("water.6-31gss.mol", "water.sto-3g.mol", "water.dzp.mol")


def _run(cmd, **kw):
    subprocess.run(cmd, check=True, **kw)


def _stale(out, deps):
    return not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out)
                                          for d in deps if os.path.exists(d))


def _link_b200():
    # rpath relative to the binary, so the tree can move (it is copied to the
    # GPU host as a whole)
    rel = os.path.relpath(LIBDIR, OUT)
    return ["-L", LIBDIR, "-l:libsimint_b200.so", "-Wl,-rpath,$ORIGIN/" + rel]


def build_driver():
    out = os.path.join(OUT, "librefdrv_b200.so")
    src = os.path.join(HERE, "refdrv.c")
    if not os.path.exists(LIB):
        return None
    if _stale(out, [src, LIB]):
        os.makedirs(OUT, exist_ok=True)
        _run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-fopenmp", "-I", INC, "-o", out, src]
             + _link_b200())
    return out


def build_examples(ref):
    skel = os.path.join(ref, "skel")
    ex = os.path.join(skel, "examples", "example1.c")
    out = os.path.join(OUT, "example1_b200")
    if os.path.exists(LIB) and _stale(out, [ex, LIB]):
        _run(["gcc", "-std=gnu11", "-O2", "-I", INC, "-o", out, ex] + _link_b200() + ["-lm"])
    # the reference's own output of the same program
    sys.path.insert(0, HERE)
    import build_reflib
    src = build_reflib.src_dir("gamess_l3")
    refout = os.path.join(OUT, "example1_ref.out")
    refbin = os.path.join(build_reflib.BUILD, "example1_ref")
    lib = build_reflib.lib_path("gamess_l3", "avx512")
    if not os.path.exists(lib):
        lib = build_reflib.lib_path("gamess_l3", "avx2")
    if os.path.exists(lib) and _stale(refout, [ex, lib]):
        stage = build_reflib.stage_dir("gamess_l3", "avx512" if "avx512" in lib else "avx2")
        _run(["gcc", "-std=gnu11", "-O2", "-I", src, "-I", stage, "-o", refbin, ex, lib,
              "-Wl,-rpath," + OUT, "-fopenmp", "-lm"])
        with open(refout, "w") as f:
            _run([refbin], stdout=f)
    # the reference's accuracy test
    tdir = os.path.join(skel, "test")
    srcs = [os.path.join(tdir, f) for f in ("test_eri.cpp", "Common.cpp", "ValeevRef.cpp")]
    out = os.path.join(OUT, "test_eri_b200")
    if os.path.exists(LIB) and _stale(out, srcs + [LIB]):
        _run(["g++", "-std=c++11", "-O2", "-fopenmp", "-w", "-Drestrict=__restrict__",
              "-I", INC, "-I", skel, "-o", out] + srcs + _link_b200() + ["-lm"])
    dat = os.path.join(OUT, "dat")
    os.makedirs(dat, exist_ok=True)
    for m in MOLS:
        s = os.path.join(tdir, "dat", m)
        if os.path.exists(s):
            shutil.copy(s, os.path.join(dat, m))


def build_all(ref=None):
    os.makedirs(OUT, exist_ok=True)
    build_driver()
    if ref and os.path.isdir(os.path.join(ref, "skel")):
        build_examples(ref)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SIMINT_REFERENCE"))
    a = ap.parse_args()
    build_all(a.ref)
    for f in sorted(os.listdir(OUT)):
        if f.endswith("_b200") or f.endswith(".out") or f == "librefdrv_b200.so":
            print(os.path.join(OUT, f))
