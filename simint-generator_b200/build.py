"""Build libsimint_b200.so for sm_100a (B200).

Steps: generate the Boys grid and the per-class kernel sources
(simint_b200/gen), compile every .cu with nvcc for sm_100a and the host
sources, and link one shared library next to this file.  Objects go to
_build/ and are rebuilt only when a source or header changed.

    python simint-generator_b200/build.py [--max-am 4] [--limit N] [-j 8]
"""

import argparse
import glob
import os
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "gen")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsimint_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# straight-line kernels for classes whose VRR elements + top quartets stay
# under this budget; larger classes use the generic kernel
DEFAULT_LIMIT = 1300

sys.path.insert(0, HERE)


def _newer(obj, deps):
    if not os.path.exists(obj):
        return False
    t = os.path.getmtime(obj)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _compile(src, obj, headers, verbose):
    if _newer(obj, [src] + headers):
        return src, 0.0, ""
    t0 = time.time()
    if src.endswith(".cu"):
        # generated kernels go without line tables (they would triple the
        # library's size); the hand-written sources keep them for profiling
        lineinfo = [] if os.path.dirname(src) == GEN else ["-lineinfo"]
        cmd = [NVCC] + ARCH + ["-O3"] + lineinfo + ["-std=c++17", "-Xcompiler", "-fPIC",
                               "-diag-suppress", "177",
                               "-I", os.path.join(REPO, "include"), "-I", CSRC,
                               "--expt-relaxed-constexpr", "--extended-lambda",
                               "-Xptxas", "-v" if verbose else "-O3",
                               "-c", src, "-o", obj]
    else:
        cmd = ["g++", "-O2", "-fPIC", "-std=c++17", "-I", os.path.join(REPO, "include"),
               "-I", CSRC, "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return src, time.time() - t0, r.stderr


def build(max_am=4, limit=DEFAULT_LIMIT, jobs=None, verbose=False, only=None):
    from simint_b200.gen.boysgrid import ensure_include
    from simint_b200.gen.sources import generate
    os.makedirs(BUILD, exist_ok=True)
    ensure_include(os.path.join(GEN, "boys_grid.inc"))
    gen_files, classes = generate(GEN, max_am=max_am, limit=limit, only=only)
    # drop stale generated kernels of classes no longer selected
    keep = set(os.path.basename(f) for f in gen_files)
    for f in glob.glob(os.path.join(GEN, "ostei_*.cu")) + glob.glob(os.path.join(GEN, "col_*.cu")):
        if os.path.basename(f) not in keep:
            os.remove(f)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) \
        + glob.glob(os.path.join(REPO, "include", "**", "*.h"), recursive=True) \
        + [os.path.join(GEN, "boys_grid.inc")]
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))) \
        + sorted(gen_files, key=lambda f: -os.path.getsize(f))
    objs = []
    jobs = jobs or os.cpu_count() or 4
    work = []
    for s in srcs:
        rel = os.path.relpath(s, CSRC).replace(os.sep, "_")
        obj = os.path.join(BUILD, rel + ".o")
        objs.append(obj)
        work.append((s, obj))
    logs = []
    # generated kernels include only the device header and the kernel table
    # (straight-line) or the column kernel's headers
    gen_headers = [os.path.join(CSRC, "ostei_device.cuh"), os.path.join(CSRC, "kernels.h")]
    col_headers = gen_headers + [os.path.join(CSRC, h) for h in ("colkern.cuh", "coop2.cuh", "cartinfo.cuh")] \
        + [os.path.join(REPO, "include", "simint_b200.h")]

    def deps(s):
        if os.path.dirname(s) != GEN:
            return headers
        return col_headers if os.path.basename(s).startswith("col_") else gen_headers

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, s, o, deps(s), verbose) for s, o in work]
        for f in futs:
            src, dt, err = f.result()
            if dt > 0:
                logs.append((src, dt, err))
    if logs or not os.path.exists(LIB) or not _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB, classes, logs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-am", type=int, default=4)
    ap.add_argument("--limit", type=int, default=DEFAULT_LIMIT)
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    t0 = time.time()
    lib, classes, logs = build(a.max_am, a.limit, a.j, a.v)
    for src, dt, err in sorted(logs, key=lambda x: -x[1]):
        print("%6.1fs %s" % (dt, os.path.basename(src)))
        if a.v and err:
            print(err)
    print("built %s (%d straight-line classes) in %.1fs" % (lib, len(classes), time.time() - t0))


if __name__ == "__main__":
    main()
