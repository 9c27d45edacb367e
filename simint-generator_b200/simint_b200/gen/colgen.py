"""CUDA emitter: the column kernel's per-class code (csrc/colkern.cuh).

The column kernel computes the Obara-Saika VRR of a unique class
(a b | c d) (a >= b, c >= d, a+b >= c+d) over a batch of NP primitive
quartets with one thread per (bra Cartesian function g_e of level
e = 0..a+b, primitive quartet): a thread owns the whole ket column of its
bra function,

    (g_e, 0 | f)^(m)   for every ket function f of levels 0..c+d,

built with the ket step of the 8-term recursion (the reference's
OSTEI_VRR_Algorithm_Base.cpp:449-469 builds the ket centre first when
c+d <= a+b; step direction: the smallest non-zero exponent of f, ties to
the right, Makowski.hpp:113-117):

    (e, f+1_y)^(m) = QC_y (e, f)^(m) + W_y (e, f)^(m+1)
                   + n_y(f)/2q [(e, f-1_y)^(m) - rho/q (e, f-1_y)^(m+1)]
                   + n_y(e)/2(p+q) (e-1_y, f)^(m+1).

The first three terms read the thread's own registers; only the last reads
another thread's column (the level below), through shared memory.  The
columns' starting values (g_e, 0|0)^(m) come from the bra-only recursion,
run beforehand for a block of up to 32 primitive quartets at once, level by
level (colkern.cuh, col_f0_block); the block's values stay in shared memory
(level-major: level e holds orders 0..L-e of its nc(e) functions) while its
batches of NP primitive quartets run the ket stages f = 1..c+d, one barrier
each: stage f reads the orders 1.. of stage f-1 that other threads stored
and stores its own for stage f+1.  The top quartets (e >= a, f >= c,
m = 0) are summed in registers across batches.

This file emits, per class, a traits struct with the class constants, the
shared-memory sizes and the straight-line stage code, plus the kernel
instantiations and their registration (colkern.cuh holds the kernel).
"""

from .emit import cname


def nc(l):
    return (l + 1) * (l + 2) // 2


def lo_h(l):
    return 0 if l <= 0 else l * (l + 1) * (l + 2) // 6


def carts(l):
    """Cartesians of level l in Psi4 order (flat order inside a level)."""
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


def pos(ijk):
    i, j, k = ijk
    l = i + j + k
    return ((l - i) * (l - i + 1)) // 2 + k


def stepdir(ijk):
    mn = min(x for x in ijk if x > 0)
    for x in (2, 1, 0):
        if ijk[x] == mn:
            return x


# variants: code -> (primitive quartets per batch, groups of threads per CTA)
COL_NP = {81: (4, 1), 82: (8, 1), 83: (4, 2)}


def col_supported(am):
    """Unique classes with a column kernel: bra depth a+b <= 6 (at most 84
    bra functions, so a batch of 8 primitive quartets stays within 1024
    threads and the register budget) and ket depth c+d <= 6."""
    a, b, c, d = am
    return (a >= b and c >= d and (a + b, a) >= (c + d, c) and a + b + c + d >= 2 and c + d <= 6
            and a + b <= 6)


def sizes(am):
    a, b, c, d = am
    E, F = a + b, c + d
    L = E + F
    nrole = lo_h(E + 1)
    # level-major bra block: level e holds orders 0..L-e of nc(e) functions
    lb = [0]
    for e in range(E + 1):
        lb.append(lb[-1] + nc(e) * (L - e + 1))
    sa = max([nc(f) * (F - f) * nrole for f in range(1, F + 1, 2)] + [0])
    sb = max([nc(f) * (F - f) * nrole for f in range(2, F + 1, 2)] + [0])
    return dict(E=E, F=F, L=L, NROLE=nrole, NTOP=lo_h(F + 1) - lo_h(c), F0B=lb[-1], LB=lb[:-1],
                SAN=sa, SBN=sb)


def emit_stages(am):
    """Device code of the ket stages of class am (template over T, NP)."""
    a, b, c, d = am
    E, F = a + b, c + d
    z = sizes(am)
    NR = z["NROLE"]
    o = []
    w = o.append
    reg = lambda f, p, m: "r%d_%d_%d" % (f, p, m)
    w("    template<typename T, int NP, typename SYNC>")
    w("    __device__ static __forceinline__ void stages(const T * __restrict__ F0, T * __restrict__ SA,")
    w("        T * __restrict__ SB, int own, int ownF, int ostr, const int (&loff)[3], const int (&loffF)[3],")
    w("        const int (&mstrF)[3], const T (&XQ)[3], const T (&YQ)[3], T Zq, const T (&kq)[KQN],")
    w("        const T (&cB)[3], bool valid, double (&acc)[NTOP], SYNC sync)")
    w("    {")
    w("        constexpr int RS = NROLE * NP;")
    # own f = 0 column, orders 0..F (from the block)
    w("        T %s;" % ", ".join(reg(0, 0, m) for m in range(F + 1)))
    w("        if(valid)")
    w("        {")
    for m in range(F + 1):
        w("            %s = F0[ownF + %d * ostr];" % (reg(0, 0, m), m))
    if c == 0:
        w("            acc[0] += (double)%s;" % reg(0, 0, 0))
    w("        }")
    for f in range(1, F + 1):
        area_in = "SA" if (f - 1) % 2 == 1 else "SB"
        area_out = "SA" if f % 2 == 1 else "SB"
        nm = F - f + 1                          # orders of block f: 0..F-f
        names = []
        body = []
        for p_, gf in enumerate(carts(f)):
            y = stepdir(gf)
            g1 = list(gf)
            g1[y] -= 1
            p1 = pos(g1)
            nA = gf[y] - 1
            if nA > 0:
                g2 = list(gf)
                g2[y] -= 2
                p2 = pos(g2)
            for m in range(nm):
                r = reg(f, p_, m)
                names.append(r)
                e = "XQ[%d] * %s" % (y, reg(f - 1, p1, m))
                e = "cfma(YQ[%d], %s, %s)" % (y, reg(f - 1, p1, m + 1), e)
                if nA > 0:
                    e = "cfma(kq[%d], cfma(Zq, %s, %s), %s)" % (nA - 1, reg(f - 2, p2, m + 1),
                                                              reg(f - 2, p2, m), e)
                # s3: (e - 1_y, f - 1_y)^(m+1) of the level below: from the
                # bra block for f = 1, else stored by stage f - 1 (orders
                # 1.. of block f - 1)
                if f == 1:
                    s3 = "F0[loffF[%d] + %d * mstrF[%d]]" % (y, m + 1, y)
                else:
                    cst = (p1 * (F - f + 1) + m) * NR
                    s3 = "%s[%d * NP + loff[%d]]" % (area_in, cst, y)
                e = "cfma(cB[%d], %s, %s)" % (y, s3, e)
                body.append("            %s = %s;" % (r, e))
                if m >= 1 and f <= F - 1:
                    body.append("            %s[%d * RS + own] = %s;" % (area_out, (p_ * (F - f) + m - 1), r))
                if m == 0 and f >= c:
                    t = lo_h(f) - lo_h(c) + p_
                    body.append("            acc[%d] += (double)%s;" % (t, r))
        w("        // stage f = %d: %d ket functions x %d orders" % (f, nc(f), nm))
        w("        T %s;" % ", ".join(names))
        w("        if(valid)")
        w("        {")
        o.extend(body)
        w("        }")
        w("        sync();")
    if F == 0:
        w("        sync();")
    w("    }")
    return o


def emit_traits(am):
    z = sizes(am)
    name = cname(am)
    o = []
    w = o.append
    w("struct ColT_%s" % name)
    w("{")
    w("    static constexpr int A0 = %d, A1 = %d, A2 = %d, A3 = %d;" % am)
    w("    static constexpr int E = %d, F = %d, L = %d;" % (z["E"], z["F"], z["L"]))
    w("    static constexpr int NROLE = %d, NTOP = %d, KQN = %d;" % (z["NROLE"], z["NTOP"],
                                                                   max(1, z["F"] - 1)))
    w("    static constexpr int F0B = %d, SAN = %d, SBN = %d;" % (z["F0B"], z["SAN"], z["SBN"]))
    o.extend(emit_stages(am))
    w("};")
    return "\n".join(o)


def col_file(am):
    name = cname(am)
    o = ['#include "../colkern.cuh"', "", "namespace {", emit_traits(am), "}", ""]
    o.append("void register_col_%s(ColTable & t)" % name)
    o.append("{")
    o.append("    ColKernels k;")
    o.append("    k.am[0] = %d; k.am[1] = %d; k.am[2] = %d; k.am[3] = %d;" % am)
    o.append("    col_fill<ColT_%s>(k);" % name)
    o.append("    t.add(k);")
    o.append("}")
    return "\n".join(o) + "\n"
