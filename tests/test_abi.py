"""The C-ABI library loads and exports every function the headers declare.

No compute call is made here (no GPU needed)."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

import simint_b200 as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            n = m.group(1)
            if n.startswith("simint_") and "static inline" not in text[max(0, m.start() - 80):m.start()]:
                names.add(n)
    # static inline helpers defined in the headers themselves
    inline = {"simint_ostei_worksize", "simint_ostei_workmem", "simint_malloc_aligned",
              "simint_free_aligned"}
    return sorted(names - inline)


def test_headers_declare_the_reference_api():
    names = declared_functions()
    for n in ["simint_init", "simint_finalize", "simint_compute_eri", "simint_compute_eri_deriv",
              "simint_create_multi_shellpair", "simint_normalize_shells", "simint_eri_workmem",
              "simint_primscreen_schwarz", "simint_cat_multi_shellpair", "simint_compute_overlap",
              "simint_compute_ke", "simint_compute_potential"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = sb.load()
    out = subprocess.run(["nm", "-D", "--defined-only", sb.LIBPATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)


def test_worksize_matches_reference_generator():
    """simint_ostei_workmem values equal the reference's WORK SIZE formula."""
    lib = sb.load()
    # (pp|pp) work sizes logged by the reference generator: 81 149 81
    exp_l1 = ((16 * 81 + 7) & ~7) + ((81 + 7) & ~7) + 8 * 149
    assert lib.simint_eri_worksize(0, 1) == exp_l1
    assert lib.simint_eri_workmem(0, 1) == 8 * exp_l1
    assert lib.simint_eri_worksize(1, 2) == ((16 * 5386 + 7) & ~7) + ((37116 + 7) & ~7) + 8 * 5801


def test_set_variant_validates_without_a_device():
    """simint_b200_set_variant accepts only variants that exist for a class
    (host-side planning; no kernel runs)."""
    lib = sb.load()
    lib.simint_init()
    am = (2, 2, 2, 2)
    assert sb.set_variant(am, 24, 0, sb.FP64, lib) == 0
    assert sb.get_variant(am, 0, sb.FP64, lib) == 24
    assert sb.get_variant(am, 0, sb.MIXED, lib) == 0          # per precision
    assert sb.set_variant(am, 23, 0, sb.FP64, lib) != 0       # no batch-3 kernel
    assert sb.set_variant(am, 99, 0, sb.FP64, lib) != 0
    assert sb.set_variant((5, 0, 0, 0), 4, 0, sb.FP64, lib) != 0
    assert sb.set_variant((4, 4, 4, 4), 1, 0, sb.FP64, lib) != 0   # no register kernel
    assert sb.set_variant((1, 1, 1, 1), 1, 1, sb.FP64, lib) != 0   # register kernels: deriv 0 only
    assert sb.set_variant(am, 0, 0, sb.FP64, lib) == 0
    assert sb.get_variant(am, 0, sb.FP64, lib) == 0


def test_ctypes_struct_layouts_match_the_headers(tmp_path):
    """The ctypes mirrors (simint_b200/capi.py) that the tests, the bench and
    the Python bindings use have the layout of include/simint/shell/shell.h:
    sizeof and every field's offsetof, from a C program built here."""
    from simint_b200.capi import SimintShell, SimintMultiShellpair
    structs = {"simint_shell": SimintShell, "simint_multi_shellpair": SimintMultiShellpair}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "simint/simint.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append('printf("%%s sizeof %%zu\\n", "%s", sizeof(struct %s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%%s %%s %%zu\\n", "%s", "%s", offsetof(struct %s, %s));'
                         % (cname, f, cname, f))
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines():
        a, b, c = line.split()
        got[(a, b)] = int(c)
    for cname, py in structs.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
