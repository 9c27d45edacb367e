"""Build recipe for the CPU oracle and the reference-built checker library.

TEST INFRASTRUCTURE ONLY.

* oracle/liboracle.so   <- oracle/ostei_oracle.c + osoei_oracle.c (our C
  restatements of the two- and one-electron integrals), plain
  gcc -O2, plus an OpenMP driver used only as the timed CPU baseline.
* oracle/_ref/libsimint_ref.so <- compiled straight from the reference's
  sources where they lie (no reference build system is run):
    skel/simint/shell/shell.c, shell_screen.c, shell_constants.c
        (pair precompute, normalisation, screening),
    skel/simint/boys/boys_shortgrid.c + boys.h (Boys grid and evaluation),
    skel/simint/osoei/osoei_*.c + recur_lookup.c (one-electron integrals),
    skel/test/ValeevRef.cpp (the reference's own long-double test oracle),
  with small glue files from oracle/ (ref_shim*.c*) and two configuration
  headers that the reference's CMake would otherwise generate
  (ostei_config.h, vectorization.h: 8-wide layout for the pair code, scalar
  layout for the Boys glue).  The reference's per-class ERI kernels (output of
  its code generator) are built separately by oracle/build_reflib.py.

Run `python oracle/build.py` (or __graft_entry__.build()).  The reference tree
is given as an argument or by $SIMINT_REFERENCE (no default), and is used only
when present.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GEN = os.path.join(REPO, "simint-generator_b200", "csrc", "gen")
REF = os.environ.get("SIMINT_REFERENCE")


def _run(cmd):
    subprocess.run(cmd, check=True)


def _ensure_boys():
    sys.path.insert(0, os.path.join(REPO, "simint-generator_b200"))
    from simint_b200.gen.boysgrid import ensure_include
    return ensure_include(os.path.join(GEN, "boys_grid.inc"))


def build_oracle_ld(force=False):
    """oracle/liboracle_ld.so: the same restatement evaluated in long double
    (-DORACLE_LONG_DOUBLE), used by the tests to measure the intrinsic
    double-precision error of ill-conditioned elements."""
    _ensure_boys()
    out = os.path.join(HERE, "liboracle_ld.so")
    srcs = [os.path.join(HERE, "ostei_oracle.c"), os.path.join(HERE, "osoei_oracle.c")]
    if not force and os.path.exists(out) and all(
            os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu11", "-DORACLE_LONG_DOUBLE",
          "-I", os.path.join(REPO, "include"), "-I", GEN, "-o", out] + srcs + ["-lm"])
    return out


def build_oracle(force=False):
    _ensure_boys()
    out = os.path.join(HERE, "liboracle.so")
    srcs = [os.path.join(HERE, "ostei_oracle.c"), os.path.join(HERE, "osoei_oracle.c"),
            os.path.join(HERE, "oracle_omp.c")]
    if not force and os.path.exists(out) and all(
            os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11",
          "-I", os.path.join(REPO, "include"), "-I", GEN,
          "-o", out] + srcs + ["-lm"])
    return out


_CFG8 = """#pragma once
#include <stdlib.h>
#define SIMINT_SIMD_LEN 8
#define SIMINT_SIMD_ALIGN 64
#define SIMINT_SIMD_ROUND(x) ((x + ((SIMINT_SIMD_LEN-1))) & (~(SIMINT_SIMD_LEN-1)))
#define SIMINT_NSHELL_SIMD (2*SIMINT_SIMD_LEN)
static inline void *simint_cfg_alloc(size_t n) { void *p = NULL; if(posix_memalign(&p, 64, n)) return NULL; return p; }
#define SIMINT_ALLOC(x) simint_cfg_alloc((x))
#define SIMINT_FREE(x) free((x))
"""

_CFG1 = """#pragma once
#include <stdlib.h>
#include "simint/vectorization/intrinsics_scalar.h"
#define SIMINT_SIMD_ROUND(x) (x)
#define SIMINT_NSHELL_SIMD (2*SIMINT_SIMD_LEN)
#define SIMINT_ALLOC(x) malloc((x))
#define SIMINT_FREE(x) free((x))
"""

_OSTEI_CFG = """#pragma once
#include <stddef.h>
#include "simint/vectorization/vectorization.h"
#define SIMINT_OSTEI_MAXAM 4
#define SIMINT_OSTEI_MAXDER 1
#define SIMINT_OSTEI_DERIV1_MAXAM 4
static inline size_t simint_ostei_worksize(int d, int l) { (void)d; (void)l; return 0; }
static inline size_t simint_ostei_workmem(int d, int l) { (void)d; (void)l; return 64; }
"""


def _write(path, text):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)


def build_ref(force=False, ref=None):
    """Compile the reference's hand-written pieces into oracle/_ref/."""
    ref = ref or REF
    if not ref:
        return None
    skel = os.path.join(ref, "skel")
    if not os.path.isdir(skel):
        return None
    _ensure_boys()
    outdir = os.path.join(HERE, "_ref")
    out = os.path.join(outdir, "libsimint_ref.so")
    if os.path.exists(out) and not force:
        return out
    inc8 = os.path.join(outdir, "include8")
    inc1 = os.path.join(outdir, "include1")
    _write(os.path.join(inc8, "simint", "vectorization", "vectorization.h"), _CFG8)
    _write(os.path.join(inc8, "simint", "ostei", "ostei_config.h"), _OSTEI_CFG)
    _write(os.path.join(inc1, "simint", "vectorization", "vectorization.h"), _CFG1)
    _write(os.path.join(inc1, "simint", "ostei", "ostei_config.h"), _OSTEI_CFG)
    objdir = os.path.join(outdir, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []

    def cc(src, inc, lang="c", extra=()):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        comp = ["gcc", "-std=gnu11"] if lang == "c" else ["g++", "-std=c++11", "-Drestrict=__restrict__"]
        _run(comp + ["-O2", "-fPIC", "-c", "-w", "-I", inc, "-I", skel,
                     "-I", os.path.join(REPO, "include"), "-I", GEN]
             + list(extra) + ["-o", obj, src])
        objs.append(obj)

    for f in ("shell/shell.c", "shell/shell_screen.c", "shell/shell_constants.c"):
        cc(os.path.join(skel, "simint", f), inc8)
    cc(os.path.join(skel, "simint", "boys", "boys_shortgrid.c"), inc1, extra=["-DSIMINT_SCALAR"])
    cc(os.path.join(HERE, "ref_shim_boys.c"), inc1, extra=["-DSIMINT_SCALAR"])
    # one-electron integrals (overlap, kinetic energy, nuclear attraction)
    # and the Cartesian lookup table they index through
    for f in ("osoei/osoei_overlap.c", "osoei/osoei_ke.c", "osoei/osoei_potential.c",
              "osoei/osoei_terms.c", "recur_lookup.c"):
        cc(os.path.join(skel, "simint", f), inc1, extra=["-DSIMINT_SCALAR"])
    cc(os.path.join(skel, "test", "ValeevRef.cpp"), inc8, lang="c++")
    cc(os.path.join(HERE, "ref_shim.cpp"), inc8, lang="c++")
    cc(os.path.join(HERE, "ref_shim_eri.c"), inc8)
    # the oracle answers the screening ERIs inside this library; compile it
    # against the reference's own struct definition (same layout)
    obj = os.path.join(objdir, "ostei_oracle_ref.o")
    _run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-c", "-w", "-I", inc8, "-I", skel,
          "-I", GEN, "-o", obj, os.path.join(HERE, "ostei_oracle.c")])
    objs.append(obj)
    _run(["g++", "-shared", "-Wl,-Bsymbolic", "-o", out] + objs + ["-lm"])
    return out


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_oracle_ld(force=True))
    print(build_ref(force=True, ref=sys.argv[1] if len(sys.argv) > 1 else None))
