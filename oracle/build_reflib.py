"""Recipe: the reference's own generated CPU library, built into oracle/_ref/.

TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; nothing in
the product links or loads it).

Simint is a code generator: C++ programs (generator/) write one C function per
angular-momentum class, driven by create.py, and the emitted C plus the
hand-written runtime (skel/simint/) is the library its users link.  This recipe
builds exactly that, without the reference's CMake:

1. the four generator programs (ostei_generator, ostei_deriv1_generator,
   ostei_vrr_generator, ostei_hrr_generator) compiled with g++ directly from
   generator/*.cpp + generator/ostei/*.cpp, once per Cartesian ordering
   (Ordering_GAMESS.cpp or Ordering_Psi4.cpp; generator/CMakeLists.txt:49-55
   picks one the same way);
2. create.py run with those programs (create.py:85-96 options) into
   oracle/_ref/build/src_<variant>/ -- it copies skel/ there and writes the
   generated sources, the file lists and ostei_config.h.in;
3. the two configuration headers CMake would write (vector_config.h with the
   vectorisation define, skel/CMakeLists.txt:51-59 and DefaultFlags.cmake;
   ostei_config.h from ostei_config.h.in with @SIMINT_MAXAM@/@SIMINT_MAXDER@,
   skel/simint/CMakeLists.txt:20-22);
4. every source of skel/simint/CMakeLists.txt:25-56 plus the generated file
   list compiled with gcc -O3, OpenMP, the vectorisation flags of
   skel/cmake/DefaultFlags_<vector>.cmake, into one shared library together
   with oracle/refdrv.c (our driver: shells and pair lists in, integrals out,
   OpenMP over bra pairs like skel/test/benchmark_eri.cpp:135-216).

Variants (name: generator ordering, inline options, max_am, max deriv):

* gamess_l3   GAMESS, all-inline (-ve/-vg/-he/-hg 100: the only generation
              that really produces GAMESS order), max_am 3, deriv 0
* psi4_l4     Psi4, default generation, max_am 4, deriv 0
* psi4_d1_l2  Psi4, default generation, max_am 2, deriv 1 (the reference's
              GAMESS deriv1 indexes through the Psi4 table, so deriv1 is
              checked in Psi4 order)

Each is compiled twice: `avx512` (SIMINT_COMMONAVX512, -mavx512f -mavx512cd
-mfma, -march=x86-64-v4) and `avx2` (SIMINT_AVX2, -mavx2 -mfma,
-march=x86-64-v3), so the library runs on whichever host it lands on
(oracle/reflib.py picks by /proc/cpuinfo).  Portable -march levels stand in
for -march=native because the library is built on one machine and run on
another.

Usage: python oracle/build_reflib.py [--ref PATH] [--only NAME] [--isa avx512|avx2]
The reference tree comes from --ref or $SIMINT_REFERENCE (no default).
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
BUILD = os.path.join(OUT, "build")      # generator, sources and objects (not needed at run time)

VARIANTS = {
    # name: (ordering, inline, max_am, deriv)
    "gamess_l3": ("GAMESS", True, 3, 0),
    "psi4_l4": ("Psi4", False, 4, 0),
    "psi4_d1_l2": ("Psi4", False, 2, 1),
}

ISAS = {
    "avx512": ("SIMINT_COMMONAVX512", ["-march=x86-64-v4", "-mavx512f", "-mavx512cd", "-mfma"]),
    "avx2": ("SIMINT_AVX2", ["-march=x86-64-v3", "-mavx2", "-mfma"]),
}

# skel/simint/CMakeLists.txt:25-56 (Fortran module left out)
RUNTIME_SOURCES = [
    "simint_init.c", "recur_lookup.c", "simint_eri.c", "simint_oneelectron.c",
    "boys/boys_shortgrid.c", "ostei/ostei_init.c", "ostei/ostei_deriv1_init.c",
    "ostei/ostei_general_vrr.c", "ostei/ostei_general_hrr.c", "ostei/ostei.c",
    "osoei/osoei_terms.c", "osoei/osoei_overlap.c", "osoei/osoei_potential.c",
    "osoei/osoei_ke.c", "shell/shell.c", "shell/shell_screen.c", "shell/shell_constants.c",
]


def _run(cmd, cwd=None, log=None):
    if log:
        with open(log, "w") as f:
            subprocess.run(cmd, check=True, cwd=cwd, stdout=f, stderr=subprocess.STDOUT)
    else:
        subprocess.run(cmd, check=True, cwd=cwd)


def build_generator(ref, ordering, jobs):
    """generator binaries for one ordering -> oracle/_ref/gen_<ordering>/"""
    gdir = os.path.join(BUILD, "gen_" + ordering.lower())
    progs = ["ostei_generator", "ostei_deriv1_generator", "ostei_vrr_generator",
             "ostei_hrr_generator"]
    if all(os.path.exists(os.path.join(gdir, p)) for p in progs):
        return gdir
    os.makedirs(os.path.join(gdir, "obj"), exist_ok=True)
    g = os.path.join(ref, "generator")
    common = [os.path.join(g, "CommandLine.cpp"), os.path.join(g, "Types.cpp"),
              os.path.join(g, "Ordering_%s.cpp" % ordering)]
    ostei = [os.path.join(g, "ostei", f) for f in (
        "OSTEI_VRR_Algorithm_Base.cpp", "OSTEI_HRR_Algorithm_Base.cpp", "OSTEI_VRR_Writer.cpp",
        "OSTEI_HRR_Writer.cpp", "OSTEI_Writer_Base.cpp", "OSTEI_Writer.cpp",
        "OSTEIDeriv1_Writer.cpp")]
    flags = ["g++", "-O2", "-std=c++11", "-w", "-I", ref]

    def obj(src):
        o = os.path.join(gdir, "obj", os.path.basename(src) + ".o")
        _run(flags + ["-c", "-o", o, src])
        return o

    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(obj, common + ostei))
        mains = list(ex.map(obj, [os.path.join(g, "ostei", p + ".cpp") for p in progs]))
    for p, m in zip(progs, mains):
        _run(["g++", "-o", os.path.join(gdir, p), m] + objs)
    return gdir


def generate(ref, name, jobs):
    """create.py output for one variant -> oracle/_ref/src_<name>/"""
    ordering, inline, max_am, deriv = VARIANTS[name]
    src = os.path.join(BUILD, "src_" + name)
    stamp = os.path.join(src, ".generated")
    if os.path.exists(stamp):
        return src
    gdir = build_generator(ref, ordering, jobs)
    if os.path.isdir(src):
        shutil.rmtree(src)
    cmd = [sys.executable, os.path.join(ref, "create.py"), "-g", gdir, "-l", str(max_am),
           "-p", str(max_am + 1), "-d", str(deriv), "-n", str(jobs)]
    if inline:
        cmd += ["-ve", "100", "-vg", "100", "-he", "100", "-hg", "100"]
    cmd.append(src)
    os.makedirs(BUILD, exist_ok=True)
    _run(cmd, log=os.path.join(BUILD, "create_%s.log" % name))
    open(stamp, "w").close()
    return src


def _config_headers(src, name, isa):
    ordering, inline, max_am, deriv = VARIANTS[name]
    stage = os.path.join(BUILD, "stage_%s_%s" % (name, isa))
    vc = os.path.join(stage, "simint", "vectorization", "vector_config.h")
    oc = os.path.join(stage, "simint", "ostei", "ostei_config.h")
    os.makedirs(os.path.dirname(vc), exist_ok=True)
    os.makedirs(os.path.dirname(oc), exist_ok=True)
    with open(vc, "w") as f:
        f.write("#pragma once\n#define %s\n" % ISAS[isa][0])
    tmpl = open(os.path.join(src, "simint", "ostei", "ostei_config.h.in")).read()
    with open(oc, "w") as f:
        f.write(tmpl.replace("@SIMINT_MAXAM@", str(max_am)).replace("@SIMINT_MAXDER@", str(deriv)))
    return stage


def src_dir(name):
    return os.path.join(BUILD, "src_" + name)


def stage_dir(name, isa):
    return os.path.join(BUILD, "stage_%s_%s" % (name, isa))


def lib_path(name, isa):
    return os.path.join(OUT, "libsimint_%s_%s.so" % (name, isa))


def compile_lib(ref, name, isa, jobs):
    out = lib_path(name, isa)
    drv = os.path.join(HERE, "refdrv.c")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(drv):
        return out
    ordering, inline, max_am, deriv = VARIANTS[name]
    src = generate(ref, name, jobs)
    stage = _config_headers(src, name, isa)
    objdir = os.path.join(BUILD, "obj_%s_%s" % (name, isa))
    os.makedirs(objdir, exist_ok=True)
    lst = open(os.path.join(src, "simint", "ostei", "gen",
                            "filelist_d%d_%d" % (deriv, max_am))).read().split()
    srcs = [os.path.join(src, "simint", f) for f in RUNTIME_SOURCES]
    srcs += [os.path.join(src, "simint", f) if os.path.sep in f or "/" in f
             else os.path.join(src, "simint", "ostei", "gen", f) for f in lst]
    # the file lists name files relative to simint/ (ostei/gen/...)
    srcs = [s if os.path.exists(s) else os.path.join(src, "simint", "ostei", "gen",
                                                     os.path.basename(s)) for s in srcs]
    flags = ["gcc", "-std=gnu11", "-O3", "-fopenmp", "-fPIC", "-w",
             "-I", src, "-I", stage] + ISAS[isa][1]

    def cc(s):
        o = os.path.join(objdir, os.path.relpath(s, src).replace(os.path.sep, "_") + ".o")
        if not (os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(s)):
            _run(flags + ["-c", "-o", o, s])
        return o

    # largest files first so the long compiles start early
    srcs = sorted(set(srcs), key=lambda s: -os.path.getsize(s))
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(cc, srcs))
    dobj = os.path.join(objdir, "refdrv.o")
    _run(flags + ["-c", "-o", dobj, drv])
    _run(["gcc", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", out, dobj] + objs + ["-lm"])
    return out


def build_all(ref, only=None, isas=("avx512", "avx2"), jobs=None):
    if ref is None or not os.path.isdir(os.path.join(ref, "skel")):
        return []
    jobs = jobs or os.cpu_count() or 1
    built = []
    for name in VARIANTS:
        if only and name != only:
            continue
        for isa in isas:
            built.append(compile_lib(ref, name, isa, jobs))
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SIMINT_REFERENCE"))
    ap.add_argument("--only", default=None)
    ap.add_argument("--isa", default=None)
    a = ap.parse_args()
    if not a.ref:
        sys.exit("give the reference tree with --ref or $SIMINT_REFERENCE")
    for p in build_all(a.ref, a.only, (a.isa,) if a.isa else ("avx512", "avx2")):
        print(p)
