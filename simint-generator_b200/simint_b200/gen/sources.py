"""Write the generated CUDA sources (one file per unique AM class).

Each file holds the straight-line device function of one unique class (see
emit.py) in its FP64 and mixed variants, thread-per-quartet and
warp-per-quartet, the __global__ wrappers for the task modes (rectangle of
simint_compute_eri, explicit task list, screened sweep), plus a registration
function.  A registry file lists them.
"""

import itertools
import os

from .emit import emit_class, unique_class, cname
from .plan import class_plan
from . import colgen

HEADER = '#include "../ostei_device.cuh"\n#include "../kernels.h"\n\n'


def unique_classes(max_am):
    out = []
    for am in itertools.product(range(max_am + 1), repeat=4):
        if unique_class(am)[0] == am:
            out.append(am)
    return out


def straight_line_ok(am, limit):
    p = class_plan(*am)
    return len(p.vrr_elements()) + p.ntop() <= limit


def kernel_file(am):
    name = cname(am)
    p = class_plan(*am)
    src64, fn64, ntop = emit_class(am, "f64")
    srcmx, fnmx, _ = emit_class(am, "mixed")
    src64w, fn64w, _ = emit_class(am, "f64", warp=True)
    srcmxw, fnmxw, _ = emit_class(am, "mixed", warp=True)
    o = [HEADER, src64, srcmx, src64w, srcmxw]
    o.append("template<int MODE, int PREC>")
    o.append("__global__ void __launch_bounds__(128) k_%s(const KernArgs a)" % name)
    o.append("{")
    o.append("    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;")
    o.append("    int iP, iQ; long long off;")
    o.append("    if(!task_of<MODE>(a, t, iP, iQ, off)) return;")
    o.append("    QuartetCtx c;")
    o.append("    make_ctx(a, iP, iQ, c);")
    o.append("    if(PREC == 1) { c.gL = %d; c.gamp = hrr_amp(c, %d, %d); }"
             % (p.L, min(am[0], am[1]), min(am[2], am[3])))
    o.append("    if(PREC == 0) %s<false>(c, a.out + off);" % fn64)
    o.append("    else %s<true>(c, a.out + off);" % fnmx)
    o.append("}")
    o.append("")
    # warp-per-quartet wrappers (rectangle and screened-sweep modes)
    o.append("template<int MODE, int PREC>")
    o.append("__global__ void __launch_bounds__(128) kw_%s(const KernArgs a)" % name)
    o.append("{")
    o.append("    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;")
    o.append("    int iP, iQ; long long off;")
    o.append("    if(!task_of<MODE>(a, t, iP, iQ, off)) return;")
    o.append("    QuartetCtx c;")
    o.append("    make_ctx(a, iP, iQ, c);")
    o.append("    if(PREC == 1) { c.gL = %d; c.gamp = hrr_amp(c, %d, %d); }"
             % (p.L, min(am[0], am[1]), min(am[2], am[3])))
    o.append("    if(PREC == 0) %s<false>(c, a.out + off);" % fn64w)
    o.append("    else %s<true>(c, a.out + off);" % fnmxw)
    o.append("}")
    o.append("")
    o.append("void register_%s(KernelTable & t)" % name)
    o.append("{")
    o.append("    ClassKernels k = {{%d, %d, %d, %d}, %d, %d, %d, %d," % (am + (p.L, ntop, p.vrr_flops(), p.hrr_flops())))
    o.append("        {{k_%s<0,0>, k_%s<0,1>}, {k_%s<1,0>, k_%s<1,1>}, {k_%s<2,0>, k_%s<2,1>}}," % ((name,) * 6))
    o.append("        {{kw_%s<0,0>, kw_%s<0,1>}, {nullptr, nullptr}, {kw_%s<2,0>, kw_%s<2,1>}}};" % ((name,) * 4))
    o.append("    t.add(k);")
    o.append("}")
    return "\n".join(o) + "\n"


def _write(path, text):
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)


def col_classes(max_am):
    """Unique classes that get a column kernel (colkern.cuh): the column
    kernel's range with L >= 4 (below that the straight-line kernels win)."""
    return [am for am in unique_classes(max_am) if colgen.col_supported(am) and sum(am) >= 4]


def generate_col(outdir, max_am=4, only=None):
    classes = col_classes(max_am)
    if only is not None:
        classes = [am for am in classes if am in only]
    files = []
    for am in classes:
        path = os.path.join(outdir, "col_%s.cu" % cname(am))
        _write(path, colgen.col_file(am))
        files.append(path)
    reg = ['#include "../colkern.cuh"', ""]
    for am in classes:
        reg.append("void register_col_%s(ColTable & t);" % cname(am))
    reg.append("")
    reg.append("void simint_b200_register_col(ColTable & t)")
    reg.append("{")
    for am in classes:
        reg.append("    register_col_%s(t);" % cname(am))
    reg.append("}")
    path = os.path.join(outdir, "col_registry.cu")
    _write(path, "\n".join(reg) + "\n")
    files.append(path)
    return files, classes


def generate(outdir, max_am=4, limit=1300, only=None):
    os.makedirs(outdir, exist_ok=True)
    classes = [am for am in unique_classes(max_am) if straight_line_ok(am, limit)]
    if only is not None:
        classes = [am for am in classes if am in only]
    files = []
    for am in classes:
        path = os.path.join(outdir, "ostei_%s.cu" % cname(am))
        text = kernel_file(am)
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as f:
                f.write(text)
        files.append(path)
    reg = ['#include "../kernels.h"', ""]
    for am in classes:
        reg.append("void register_%s(KernelTable & t);" % cname(am))
    reg.append("")
    reg.append("void simint_b200_register_generated(KernelTable & t)")
    reg.append("{")
    for am in classes:
        reg.append("    register_%s(t);" % cname(am))
    reg.append("}")
    path = os.path.join(outdir, "ostei_registry.cu")
    text = "\n".join(reg) + "\n"
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)
    files.append(path)
    cfiles, _ = generate_col(outdir, max_am=max_am, only=only)
    return files + cfiles, classes
