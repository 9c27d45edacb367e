"""CUDA emitter: straight-line, register-resident ERI kernels per AM class.

For a unique class (a b | c d) (a >= b, c >= d, a+b >= c+d, and a >= c when
a+b == c+d -- the reference's notion of a unique quartet,
generator/ostei/OSTEI_GeneratorInfo.hpp:42-55) we emit one __device__
function that computes a whole shell quartet in one thread:

  for every bra primitive i, ket primitive j that survives screening:
      set-up (p+q, PQ, alpha, 1/p, 1/q, ...)     OSTEI_Writer.cpp:586-683
      Boys F_0..F_L, times the pair prefactors    OSTEI_Writer.cpp:683-702
      VRR, straight-line, minimal (quartet, m) set   plan.ClassPlan.vrr_elements
      accumulate the top quartets in registers  (contraction)
  HRR on the contracted top quartets, straight-line   plan.ClassPlan.hrr_elements
  store through an index table (ordering and A<->B / C<->D / bra<->ket
  permutation are runtime choices, so every requested class is served by
  the kernel of its unique class).

Two arithmetic variants are emitted: FP64 throughout, and "mixed", whose VRR
runs in FP32 for primitive quartets that pass the Schwarz-bound gate (see
csrc/ostei_device.cuh) and in FP64 otherwise; Boys, prefactors, contraction
and HRR stay FP64 in both.
"""

from .plan import class_plan, TAGS
from .ordering import ncart


def unique_class(am):
    """Canonical unique class for a requested class, and the role swaps.

    Returns (U, swap_bra, swap_ket, swap_pq): U is computed with the bra role
    taken by Q when swap_pq, and with the functions inside the bra (ket) role
    pair exchanged when swap_bra (swap_ket)."""
    a, b, c, d = am
    sb = a < b
    if sb:
        a, b = b, a
    sk = c < d
    if sk:
        c, d = d, c
    spq = (a + b, a) < (c + d, c)
    if spq:
        a, b, c, d = c, d, a, b
        sb, sk = sk, sb
    return (a, b, c, d), sb, sk, spq


def is_unique(am):
    return unique_class(am)[0] == tuple(am)


def cname(am, deriv=0):
    s = "spdfghik"
    base = "%s%s%s%s" % tuple(s[x] for x in am)
    return base if deriv == 0 else base + "_d1"


class _Names:
    def __init__(self):
        self.map = {}
        self.n = 0

    def get(self, key):
        if key not in self.map:
            self.map[key] = "t%d" % self.n
            self.n += 1
        return self.map[key]


def _fmt_int(n):
    return "%d.0" % n


def emit_class(am, prec="f64", warp=False):
    """Return CUDA source text for the device function of unique class am.

    prec: "f64" or "mixed".  warp: the function runs on a whole warp for one
    shell quartet -- lanes take the (bra, ket) primitive pairs k = lane,
    lane + 32, ... (no divergence between quartets of different contraction
    depth), the top accumulators are summed over the warp by a butterfly,
    and lane 0 does the HRR and the stores."""
    p = class_plan(*am)
    assert p.deriv == 0
    name = cname(am)
    L = p.L
    vrr = p.vrr_elements()
    hrr = p.hrr_elements()
    tops = [t[:4] for t in p.tops]          # untagged for deriv 0
    ntop = len(tops)
    topidx = {t: k for k, t in enumerate(tops)}
    o = []
    w = o.append
    w("// ---- class (%s) : L=%d, %d top quartets, %d VRR elements, %d HRR steps"
      % (name, L, ntop, len(vrr), sum(1 for _, r in hrr if r is not None)))
    fn = "ostei_%s_%s%s" % (name, prec, "_w" if warp else "")
    # a class without recursion (L = 0) has no VRR to run in FP32
    mixed = prec == "mixed" and L > 0
    w("template<bool MIXED_GATE>")
    w("__device__ __forceinline__ void %s(const QuartetCtx& c0, double* __restrict__ out)" % fn)
    w("{")
    w("    QuartetCtx c = c0;")
    if mixed:
        # the gate bounds the error of one integral: each of the shell
        # quartet's primitive quartets may take gate / (their number)
        w("    if(MIXED_GATE)")
        w("    {")
        w("        c.gL = %d;" % L)
        w("        c.gamp = hrr_amp(c, %d, %d);" % (min(am[0], am[1]), min(am[2], am[3])))
        w("        c.gate = c0.gate / (double)max(1, (c.bi1 - c.bi0) * (c.kj1 - c.kj0));")
        w("    }")
    for k in range(ntop):
        w("    double acc%d = 0.0;" % k)
    if mixed:
        w("    unsigned nlow = 0;            // primitive quartets run in FP32")
    if warp:
        w("    const int lane = threadIdx.x & 31;")
        w("    const int nj = c.kj1 - c.kj0, ncand = (c.bi1 - c.bi0) * nj;")
        w("    // k / nj as a multiply-high, exact while k * nj < 2^32")
        w("    const unsigned long long njinv = (1ull << 32) / (unsigned)max(nj, 1) + 1ull;")
        w("    const bool fastdiv = (long long)ncand * nj < (1LL << 32);")
        w("    for(int k = lane; k < ncand; k += 32)")
        w("    {")
        w("        const int kq = fastdiv ? (int)(((unsigned long long)k * njinv) >> 32) : k / nj;")
        w("        const int i = c.bi0 + kq, j = c.kj0 + (k - kq * nj);")
        w("        const BraPrim bp = load_bra_prim(c, i);")
        w("        if(c.check && bp.skip) continue;")
        w("        {")
    else:
        w("    for(int i = c.bi0; i < c.bi1; ++i)")
        w("    {")
        w("        const BraPrim bp = load_bra_prim(c, i);")
        w("        if(c.check && bp.skip) continue;")
        w("        for(int j = c.kj0; j < c.kj1; ++j)")
        w("        {")
    w("            PrimSetup s;")
    w("            if(!prim_setup(c, bp, j, s)) continue;")
    w("            double F[%d];" % (L + 1))
    w("            boys_split<%d>(c.boys, s.T, F);" % L)
    w("            #pragma unroll")
    w("            for(int n = 0; n <= %d; n++) F[n] *= s.prefac;" % L)

    def emit_vrr(T, fma_, suffix):
        """Emit the VRR in type T (double or float)."""
        names = _Names()
        lines = []
        # coefficient constants n/2p etc. are formed lazily
        consts = {}

        def const(kind, n):
            key = (kind, n)
            if key not in consts:
                base = {"2p": "s.oo2p", "2q": "s.oo2q", "2pq": "s.oo2pq"}[kind] + suffix
                nm = "k%s_%d" % (kind, n)
                if n == 1:
                    lines.append("            const %s %s = %s;" % (T, nm, base))
                else:
                    lit = ("%d.0f" % n) if T == "float" else _fmt_int(n)
                    lines.append("            const %s %s = %s * %s;" % (T, nm, lit, base))
                consts[key] = nm
            return consts[key]

        for (q, m), rule in vrr:
            var = names.get((q, m))
            if rule is None:
                src = "F[%d]" % m if T == "double" else "(float)F[%d]" % m
                lines.append("            const %s %s = %s;" % (T, var, src))
                continue
            st, x, srcs, ints = rule
            if st in (0, 1):
                X = ("s.PA%s" if st == 0 else "s.PB%s") % "xyz"[x]
                Y = "s.aopPQ%s" % "xyz"[x]
                Z = "s.a_over_p"
                h1, h2 = "2p", "2pq"
            else:
                X = ("s.QC%s" if st == 2 else "s.QD%s") % "xyz"[x]
                Y = "s.aoqPQ%s" % "xyz"[x]
                Z = "s.a_over_q"
                h1, h2 = "2q", "2pq"
            X += suffix
            Y += suffix
            Z += suffix
            n0, n1, n2, n3 = ints
            expr = "%s * %s" % (X, names.get(srcs[0]))
            if srcs[1] is not None:
                expr = "%s(%s, %s, %s)" % (fma_, Y, names.get(srcs[1]), expr)
            if srcs[2] is not None:
                k0 = const(h1, n0)
                expr = "%s(%s, %s(%s, %s, %s), %s)" % (fma_, k0, fma_, Z, names.get(srcs[3]),
                                                        names.get(srcs[2]), expr)
            if srcs[4] is not None:
                k1 = const(h1, n1)
                expr = "%s(%s, %s(%s, %s, %s), %s)" % (fma_, k1, fma_, Z, names.get(srcs[5]),
                                                        names.get(srcs[4]), expr)
            if srcs[6] is not None:
                k2 = const(h2, n2)
                expr = "%s(%s, %s, %s)" % (fma_, k2, names.get(srcs[6]), expr)
            if srcs[7] is not None:
                k3 = const(h2, n3)
                expr = "%s(%s, %s, %s)" % (fma_, k3, names.get(srcs[7]), expr)
            lines.append("            const %s %s = %s;" % (T, var, expr))
        # accumulate the tops (m = 0)
        for t in tops:
            v = names.get((t, 0))
            k = topidx[t]
            if T == "double":
                lines.append("            acc%d += %s;" % (k, v))
            else:
                lines.append("            acc%d += (double)%s;" % (k, v))
        return lines

    if not mixed:
        o.extend(emit_vrr("double", "fma", ""))
    else:
        w("            if(MIXED_GATE && s.lowprec)")
        w("            {")
        w("            s.make_f32();")
        w("            nlow++;")
        o.extend(emit_vrr("float", "fmaf", "_f"))
        w("            }")
        w("            else")
        w("            {")
        o.extend(emit_vrr("double", "fma", ""))
        w("            }")
    w("        }")
    w("    }")
    if mixed:
        # FP32 primitive quartets of the converged threads, one atomic each
        w("    if(MIXED_GATE && c.fp32_count)")
        w("    {")
        w("        const unsigned m = __activemask();")
        w("        const unsigned tot = __reduce_add_sync(m, nlow);")
        w("        if((int)(threadIdx.x & 31) == __ffs(m) - 1 && tot)")
        w("            atomicAdd(c.fp32_count, (unsigned long long)tot);")
        w("    }")
    if warp:
        # butterfly sums over the warp (every lane ends with the totals)
        w("    #pragma unroll")
        w("    for(int sh = 16; sh > 0; sh >>= 1)")
        w("    {")
        for k in range(ntop):
            w("        acc%d += __shfl_xor_sync(0xffffffffu, acc%d, sh);" % (k, k))
        w("    }")
        w("    if(lane != 0) return;")
    # HRR
    hn = {}
    for q, rule in hrr:
        key = q[:4]
        if rule is None:
            hn[q] = "acc%d" % topidx[key]
            continue
    if any(r is not None for _, r in hrr):
        w("    const double ABx = c.AB[0], ABy = c.AB[1], ABz = c.AB[2];")
        w("    const double CDx = c.CD[0], CDy = c.CD[1], CDz = c.CD[2];")
    cnt = 0
    for q, rule in hrr:
        if rule is None:
            continue
        s0, s1, x, sign, side = rule
        X = ("AB" if side == 0 else "CD") + "xyz"[x]
        if sign < 0:
            X = "-" + X
        nm = "h%d" % cnt
        cnt += 1
        w("    const double %s = fma(%s, %s, %s);" % (nm, X, hn[s1], hn[s0]))
        hn[q] = nm
    # store
    finals = p.final_quartets()
    w("    const unsigned short* __restrict__ oi = c.oidx;")
    for n, fq in enumerate(finals):
        w("    out[oi[%d]] = %s;" % (n, hn[fq + ("",)]))
    w("}")
    w("")
    return "\n".join(o), fn, ntop


def class_stats(am):
    p = class_plan(*am)
    return dict(L=p.L, ntop=p.ntop(), nvrr=len(p.vrr_elements()),
                vrr_flops=p.vrr_flops(), hrr_flops=p.hrr_flops())
