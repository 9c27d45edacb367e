"""Recurrence planner for one angular-momentum class of ERIs.

This module restates, in our own code, the plan that Simint's generator makes
for a class (a b | c d):

* HRR (horizontal recurrence, contracted integrals):
  generator/ostei/OSTEI_HRR_Algorithm_Base.cpp:160-283 and the Makowski doublet
  step generator/ostei/Makowski.hpp:17-82.  The bra moves I->J unless
  am[0] < am[1] (then J->I); the ket moves K->L unless am[2] < am[3]
  (OSTEI_HRR_Algorithm_Base.cpp:164-172, taken from the lexicographically
  largest target).  The AM-level order prefers ket steps for the final
  quartets, so bra steps on the top set run first
  (OSTEI_HRR_Algorithm_Base.cpp:42-96).
* VRR (vertical recurrence, primitive integrals):
  generator/ostei/OSTEI_VRR_Algorithm_Base.cpp:289-469 with the 8-source
  step of Makowski.hpp:87-242.  The centre order is [3,2,1,0] stably sorted by
  the maximum AM of that centre over the top quartets
  (OSTEI_VRR_Algorithm_Base.cpp:449-469); a quartet is reduced on the first
  centre in that order that carries AM, in the xyz direction of its smallest
  non-zero exponent, ties going to the right-most one (Makowski.hpp:113-117).
* deriv=1 targets: the "missing" centre is the first with maximal AM and is
  recovered by translational invariance
  (generator/ostei/ostei_deriv1_generator.cpp:97-123).

Everything here is element level (one Cartesian quartet and one auxiliary
order m at a time); the emitters turn these plans into straight-line CUDA or
into tables for the cooperative kernel.
"""

from functools import lru_cache

from .ordering import ncart, psi4_order, order as cart_order, cart_index

I, J, K, L = 0, 1, 2, 3
BRA, KET = 0, 1
TAGS = ("", "2a", "2b", "2c", "2d")


def stepdir(g):
    """xyz index to recur on: smallest non-zero exponent, right-most on ties."""
    m = min(x for x in g if x > 0)
    for idx in (2, 1, 0):
        if g[idx] == m:
            return idx
    raise ValueError(g)


def down(g, x, n=1):
    return tuple(v - n if i == x else v for i, v in enumerate(g))


def up(g, x, n=1):
    return tuple(v + n if i == x else v for i, v in enumerate(g))


def valid(g):
    return min(g) >= 0


def gaussians(l):
    """All Cartesians of AM l (canonical Psi4 order; order is irrelevant here)."""
    return psi4_order(l)


# ---------------------------------------------------------------------------
# HRR
# ---------------------------------------------------------------------------

def doublet_step(d, steptype):
    """One HRR doublet step (Makowski.hpp:26-82).

    For J/L steps (moving I->J, K->L):   (a,b) = (a+1i, b-1i) + X_i (a, b-1i)
    For I/K steps (moving J->I, L->K):   (a,b) = (a-1i, b+1i) - X_i (a-1i, b)
    Returns (src0, src1, xyz, sign).
    """
    left, right = d
    if steptype in (J, L):
        x = stepdir(right)
        common = down(right, x)
        src0 = (up(left, x), common)
        src1 = (left, common)
        return src0, src1, x, +1
    x = stepdir(left)
    common = down(left, x)
    src0 = (common, up(right, x))
    src1 = (common, right)
    return src0, src1, x, -1


def stepping_am(d, steptype):
    left, right = d
    return sum(right) if steptype in (J, L) else sum(left)


def solve_doublets(initial, steptype):
    """HRRDoubletLoop_ (OSTEI_HRR_Algorithm_Base.cpp:99-136): step every doublet
    whose stepping side carries AM; the rest are top doublets."""
    steps = {}
    work = [d for d in initial if stepping_am(d, steptype) > 0]
    while work:
        new = []
        for d in work:
            if d in steps:
                continue
            s0, s1, x, sign = doublet_step(d, steptype)
            steps[d] = (s0, s1, x, sign)
            for s in (s0, s1):
                if s not in steps and stepping_am(s, steptype) > 0:
                    new.append(s)
        work = new
    return steps


def doublet_am(d):
    return (sum(d[0]), sum(d[1]))


class HRRPlan:
    """HRR plan for a set of target quartet AMs (with derivative tags)."""

    def __init__(self, targets):
        # targets: iterable of (a, b, c, d, tag)
        targets = sorted(set(targets), key=lambda t: (t[:4], t[4]))
        highest = targets[-1]
        self.brastep = J if highest[0] >= highest[1] else I
        self.ketstep = L if highest[2] >= highest[3] else K

        initkets, initbras = [], []
        for t in targets:
            initkets += [(g1, g2) for g1 in gaussians(t[2]) for g2 in gaussians(t[3])]
            initbras += [(g1, g2) for g1 in gaussians(t[0]) for g2 in gaussians(t[1])]
        self.ketsteps = solve_doublets(initkets, self.ketstep)
        self.brasteps = solve_doublets(initbras, self.brastep)
        allketam = {doublet_am(d) for d in self.ketsteps}
        allbraam = {doublet_am(d) for d in self.brasteps}

        # AM-level order and top AMs (OSTEI_HRR_Algorithm_Base.cpp:42-96)
        self.order = []          # list of (a,b,c,d,tag) in evaluation order
        self.stepmap = {}        # qam -> BRA/KET
        self.topqam = set()

        def ket_req(dam):
            x, y = dam
            if self.ketstep == L:
                return [(x + 1, y - 1), (x, y - 1)]
            return [(x - 1, y + 1), (x - 1, y)]

        def bra_req(dam):
            x, y = dam
            if self.brastep == J:
                return [(x + 1, y - 1), (x, y - 1)]
            return [(x - 1, y + 1), (x - 1, y)]

        def add(ams):
            new, done = [], []
            for q in ams:
                if q in self.order:
                    continue
                bam, kam = (q[0], q[1]), (q[2], q[3])
                if bam not in allbraam and kam not in allketam:
                    self.topqam.add(q)
                    continue
                if kam in allketam:
                    self.stepmap[q] = KET
                    for r in ket_req(kam):
                        new.append((q[0], q[1], r[0], r[1], q[4]))
                else:
                    self.stepmap[q] = BRA
                    for r in bra_req(bam):
                        new.append((r[0], r[1], q[2], q[3], q[4]))
                done.append(q)
            if new:
                add(sorted(set(new), key=lambda t: (t[:4], t[4])))
            for q in done:
                if q not in self.order:
                    self.order.append(q)

        add(targets)
        self.targets = targets

    def top_quartets(self):
        """All Cartesian quartets (A,B,C,D,tag) of the top AMs."""
        out = []
        for q in sorted(self.topqam, key=lambda t: (t[:4], t[4])):
            for ga in gaussians(q[0]):
                for gb in gaussians(q[1]):
                    for gc in gaussians(q[2]):
                        for gd in gaussians(q[3]):
                            out.append((ga, gb, gc, gd, q[4]))
        return out

    def rule(self, quartet):
        """How one contracted Cartesian quartet (A,B,C,D,tag) is formed.

        Returns None for a top quartet, else (src0, src1, xyz, sign, side) with
        side BRA (uses AB) or KET (uses CD)."""
        A, B, C, D, tag = quartet
        qam = (sum(A), sum(B), sum(C), sum(D), tag)
        if qam in self.topqam:
            return None
        side = self.stepmap[qam]
        if side == KET:
            s0, s1, x, sign = self.ketsteps[(C, D)]
            return ((A, B) + s0 + (tag,), (A, B) + s1 + (tag,), x, sign, KET)
        s0, s1, x, sign = self.brasteps[(A, B)]
        return (s0 + (C, D, tag), s1 + (C, D, tag), x, sign, BRA)


# ---------------------------------------------------------------------------
# VRR
# ---------------------------------------------------------------------------

def vrr_center_order(topquartets):
    """Centre order for the VRR (OSTEI_VRR_Algorithm_Base.cpp:449-469)."""
    qmax = [0, 0, 0, 0]
    for q in topquartets:
        for c in range(4):
            qmax[c] = max(qmax[c], sum(q[c]))
    order = [3, 2, 1, 0]
    order.sort(key=lambda c: qmax[c])   # Python's sort is stable
    return tuple(order)


# Coefficient kinds of the 8-term VRR step (OSTEI_VRR_Writer.cpp:33-130)
#   t  = X[x]*s0 + Y[x]*s1 + n0*H1*(s2 + Z*s3) + n1*H1*(s4 + Z*s5)
#        + n2*H2*s6 + n3*H2*s7
# bra step (I,J): X = PA or PB, Y = -a/p*PQ, Z = -a/p, H1 = 1/2p, H2 = 1/2(p+q)
# ket step (K,L): X = QC or QD, Y = +a/q*PQ, Z = -a/q, H1 = 1/2q, H2 = 1/2(p+q)

def vrr_rule(quartet, m, center_order):
    """Makowski 8-source VRR step for one primitive quartet (Makowski.hpp:87-242).

    quartet: (A,B,C,D); returns None for (ss|ss) else
    (steptype, xyz, srcs, ints) where srcs is a list of 8 entries
    ((A,B,C,D), m) or None, and ints = (n0, n1, n2, n3)."""
    if all(sum(g) == 0 for g in quartet):
        return None
    st = next(c for c in center_order if sum(quartet[c]) > 0)
    A, B, C, D = quartet
    x = stepdir(quartet[st])
    q = list(quartet)

    def mk(changes, mm):
        qq = list(q)
        for c, n in changes:
            qq[c] = down(qq[c], x, n)
        if not all(valid(g) for g in qq):
            return None
        return (tuple(qq), mm)

    if st == I:
        srcs = [mk([(I, 1)], m), mk([(I, 1)], m + 1),
                mk([(I, 2)], m), mk([(I, 2)], m + 1),
                mk([(I, 1), (J, 1)], m), mk([(I, 1), (J, 1)], m + 1),
                mk([(I, 1), (K, 1)], m + 1), mk([(I, 1), (L, 1)], m + 1)]
        ints = (A[x] - 1, B[x], C[x], D[x])
    elif st == J:
        srcs = [mk([(J, 1)], m), mk([(J, 1)], m + 1),
                mk([(I, 1), (J, 1)], m), mk([(I, 1), (J, 1)], m + 1),
                mk([(J, 2)], m), mk([(J, 2)], m + 1),
                mk([(J, 1), (K, 1)], m + 1), mk([(J, 1), (L, 1)], m + 1)]
        ints = (A[x], B[x] - 1, C[x], D[x])
    elif st == K:
        srcs = [mk([(K, 1)], m), mk([(K, 1)], m + 1),
                mk([(K, 2)], m), mk([(K, 2)], m + 1),
                mk([(K, 1), (L, 1)], m), mk([(K, 1), (L, 1)], m + 1),
                mk([(I, 1), (K, 1)], m + 1), mk([(J, 1), (K, 1)], m + 1)]
        ints = (C[x] - 1, D[x], A[x], B[x])
    else:
        srcs = [mk([(L, 1)], m), mk([(L, 1)], m + 1),
                mk([(K, 1), (L, 1)], m), mk([(K, 1), (L, 1)], m + 1),
                mk([(L, 2)], m), mk([(L, 2)], m + 1),
                mk([(I, 1), (L, 1)], m + 1), mk([(J, 1), (L, 1)], m + 1)]
        ints = (C[x], D[x] - 1, A[x], B[x])
    # a pair (s2,s3) / (s4,s5) only contributes when both members exist
    if srcs[2] is None or srcs[3] is None:
        srcs[2] = srcs[3] = None
    if srcs[4] is None or srcs[5] is None:
        srcs[4] = srcs[5] = None
    return st, x, srcs, ints


# ---------------------------------------------------------------------------
# Whole-class plan
# ---------------------------------------------------------------------------

def deriv1_targets(am):
    """HRR targets of the deriv=1 kernel (ostei_deriv1_generator.cpp:97-123)."""
    mx = max(am)
    missing = am.index(mx)
    tgts = []
    for i in range(4):
        if i == missing:
            continue
        p = list(am); p[i] += 1
        tgts.append(tuple(p) + (TAGS[i + 1],))
        mm = list(am); mm[i] -= 1
        if mm[i] >= 0:
            tgts.append(tuple(mm) + ("",))
    return missing, tgts


@lru_cache(maxsize=None)
def class_plan(a, b, c, d, deriv=0):
    return ClassPlan((a, b, c, d), deriv)


class ClassPlan:
    def __init__(self, am, deriv=0):
        self.am = tuple(am)
        self.deriv = deriv
        self.L = sum(am) + deriv
        if deriv == 0:
            self.missing = None
            self.hrr = HRRPlan([self.am + ("",)])
        else:
            self.missing, tg = deriv1_targets(self.am)
            self.hrr = HRRPlan(tg)
        self.tops = self.hrr.top_quartets()
        untagged = sorted({t[:4] for t in self.tops})
        self.vrr_tops = untagged
        self.center_order = vrr_center_order(untagged)
        self._vrr = None

    # -- VRR closure ------------------------------------------------------
    def vrr_elements(self):
        """Topologically ordered list of needed (quartet, m) with their rules."""
        if self._vrr is not None:
            return self._vrr
        seen = {}
        out = []
        stack = [((q, 0), False) for q in reversed(self.vrr_tops)]
        while stack:
            key, expanded = stack.pop()
            if key in seen:
                continue
            q, m = key
            rule = vrr_rule(q, m, self.center_order)
            if expanded or rule is None:
                seen[key] = rule
                out.append((key, rule))
                continue
            stack.append((key, True))
            for s in rule[2]:
                if s is not None and s not in seen:
                    stack.append((s, False))
        self._vrr = out
        return out

    def vrr_flops(self):
        """FLOPs of the minimal VRR (FMA = 2, mul = 1), counted like Appendix A."""
        f = 0
        for key, rule in self.vrr_elements():
            if rule is None:
                continue
            srcs = rule[2]
            f += 1                      # X*s0
            f += 2 if srcs[1] else 0    # fma Y*s1
            f += 4 if srcs[2] else 0    # fma(H, fma(Z,s3,s2))
            f += 4 if srcs[4] else 0
            f += 2 if srcs[6] else 0
            f += 2 if srcs[7] else 0
        return f

    # -- HRR closure ------------------------------------------------------
    def final_quartets(self):
        """Cartesian quartets of the final output, in Psi4 order."""
        a, b, c, d = self.am
        return [(ga, gb, gc, gd) for ga in psi4_order(a) for gb in psi4_order(b)
                for gc in psi4_order(c) for gd in psi4_order(d)]

    def hrr_needed_targets(self):
        if self.deriv == 0:
            return [q + ("",) for q in self.final_quartets()]
        need = []
        for (A, B, C, D) in self.final_quartets():
            for ctr in range(4):
                if ctr == self.missing:
                    continue
                g = [A, B, C, D]
                for x in range(3):
                    gp = list(g); gp[ctr] = up(g[ctr], x)
                    need.append(tuple(gp) + (TAGS[ctr + 1],))
                    if g[ctr][x] > 0:
                        gm = list(g); gm[ctr] = down(g[ctr], x)
                        need.append(tuple(gm) + ("",))
        return need

    def hrr_elements(self):
        """Topologically ordered contracted quartets with their HRR rule."""
        seen = {}
        out = []
        stack = [(q, False) for q in reversed(self.hrr_needed_targets())]
        while stack:
            q, expanded = stack.pop()
            if q in seen:
                continue
            rule = self.hrr.rule(q)
            if expanded or rule is None:
                seen[q] = rule
                out.append((q, rule))
                continue
            stack.append((q, True))
            for s in rule[:2]:
                if s not in seen:
                    stack.append((s, False))
        return out

    def hrr_flops(self):
        return sum(2 for q, r in self.hrr_elements() if r is not None)

    def ntop(self):
        return len(self.tops)

    # -- reference work-size bookkeeping -----------------------------------
    def reference_worksize(self):
        """(bcont, prim, cont) element counts as logged by the reference
        generator ("WORK SIZE", OSTEI_Writer.cpp:348-368,753)."""
        bcont = sum(ncart(q[0]) * ncart(q[1]) * ncart(q[2]) * ncart(q[3])
                    for q in self.hrr.topqam)
        mreq = {}
        for (q, m), rule in self.vrr_elements():
            qam = tuple(sum(g) for g in q)
            mreq[qam] = max(mreq.get(qam, 0), m)
            if rule is not None:
                for s in rule[2]:
                    if s is not None:
                        sam = tuple(sum(g) for g in s[0])
                        mreq[sam] = max(mreq.get(sam, 0), s[1])
        mreq.setdefault((0, 0, 0, 0), 0)
        prim = sum(ncart(q[0]) * ncart(q[1]) * ncart(q[2]) * ncart(q[3]) * (m + 1)
                   for q, m in mreq.items())
        final = self.am + ("",)
        cont = 0
        for q in self.hrr.order:
            if q in self.hrr.topqam:
                continue
            if self.deriv > 0 or q != final:
                cont += ncart(q[0]) * ncart(q[1]) * ncart(q[2]) * ncart(q[3])
        return bcont, prim, cont


def out_index(quartet, am, ordering):
    """Offset of a Cartesian quartet inside one shell quartet's output block."""
    a, b, c, d = am
    A, B, C, D = quartet
    ia, ib = cart_index(A, ordering), cart_index(B, ordering)
    ic, id_ = cart_index(C, ordering), cart_index(D, ordering)
    return ((ia * ncart(b) + ib) * ncart(c) + ic) * ncart(d) + id_
