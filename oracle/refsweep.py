"""The reference's generated CPU library over the rows of a screened sweep.

TEST INFRASTRUCTURE ONLY: bench.py's reference arm and cpu_baseline leg, and
tests/, use it; the product never does.

A screened sweep (the workload of the B200 library's simint_b200_basis_*
calls) is, per AM class, a list of rows: one bra shell pair against the
ket shell pairs of one pair class whose Schwarz bound survives.  The rule,
restated here so the reference can be run over the same rows without the
B200 library:

* shells of am <= max_am are grouped by am; pair classes (la >= lb) hold the
  pairs (i in am la, j in am lb), j <= i when la == lb, in that order;
* each pair's bound Q_ab = sqrt(max |(ab|ab)|) (simint_shellscreen_schwarz,
  skel/simint/shell/shell_screen.c:48-83, here computed by the reference
  library itself); pairs sorted by decreasing Q (stable);
* quartet classes: pair classes ordered by (la + lb, la) descending, bra
  class X before or equal to ket class Y in that order; for the bra pairs of
  X in sorted order, the kets are the sorted pairs of Y with
  Q_bra * Q_ket >= tol (a prefix), and at most the first bra-position + 1
  when X == Y; rows with no ket are dropped;
* a stride sample keeps rows offset, offset + stride, ... of every class.

A row runs as simint_compute_eri(P, Q) with P the bra pair alone and Q the
ket class's sorted pair list clipped to the row's ket count (nshell12_clip),
both built by the reference with SIMINT_SCREEN_SCHWARZ (primitive screening at
the same tolerance, as the sweep does).
"""

import importlib.util
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SCREEN_SCHWARZ = 1


def workloads():
    """simint_b200/workloads.py loaded by path (plain numpy; the package
    itself, and with it the B200 library, stays unloaded)."""
    path = os.path.join(REPO, "simint-generator_b200", "simint_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("sb200_workloads", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def pair_classes(shells, max_am):
    byam = [[] for _ in range(max_am + 1)]
    for k, s in enumerate(shells):
        if s[0] <= max_am:
            byam[s[0]].append(k)
    pcs = []
    for la in range(max_am + 1):
        for lb in range(la + 1):
            if not byam[la] or not byam[lb]:
                continue
            pairs = [(i, j) for i in byam[la] for j in byam[lb] if not (la == lb and j > i)]
            pcs.append({"la": la, "lb": lb, "pairs": np.array(pairs, dtype=np.int32)})
    return pcs


def sweep_rows(R, shells, tol, max_am, threads=None):
    """Pair classes (with sorted order and bounds) and quartet classes
    (with their rows) of the screened sweep, bounds from reference R."""
    pcs = pair_classes(shells, max_am)
    for pc in pcs:
        q = np.sqrt(R.schwarz(pc["pairs"], threads))
        pc["Q"] = q
        pc["order"] = np.argsort(-q, kind="stable")
    cls = sorted(range(len(pcs)), key=lambda x: (pcs[x]["la"] + pcs[x]["lb"], pcs[x]["la"]),
                 reverse=True)
    qcs = []
    for xi in range(len(cls)):
        for yi in range(xi, len(cls)):
            X, Y = pcs[cls[xi]], pcs[cls[yi]]
            qy = Y["Q"][Y["order"]]
            qbs = X["Q"][X["order"]]
            ny = len(qy)
            if tol > 0.0:
                # kets with qb * qy >= tol: a prefix of the decreasing list;
                # the division's rounding is corrected with exact products
                with np.errstate(divide="ignore"):
                    cut = np.searchsorted(-qy, -(tol / np.maximum(qbs, 1e-300)), side="right")
                for b in range(len(qbs)):
                    c = int(cut[b])
                    while c > 0 and qbs[b] * qy[c - 1] < tol:
                        c -= 1
                    while c < ny and qbs[b] * qy[c] >= tol:
                        c += 1
                    cut[b] = c
            else:
                cut = np.full(len(qbs), ny)
            if cls[xi] == cls[yi]:
                cut = np.minimum(cut, np.arange(1, len(qbs) + 1))
            rows = [(int(ip), int(c)) for ip, c in zip(X["order"], cut) if c > 0]
            if rows:
                qcs.append({"am": (X["la"], X["lb"], Y["la"], Y["lb"]), "bx": cls[xi],
                            "ky": cls[yi], "rows": rows})
    return pcs, qcs


def ncart(l):
    return (l + 1) * (l + 2) // 2


class RefSweep:
    """Reference pair sets for the sampled rows of a sweep, ready to time."""

    def __init__(self, R, shells, tol, max_am, stride=1, offset=0, threads=None):
        self.R = R
        self.tol = tol
        t0 = time.time()
        R.set_shells(shells)
        self.pcs, self.qcs = sweep_rows(R, shells, tol, max_am, threads)
        screen = SCREEN_SCHWARZ if tol > 0.0 else 0
        # ket pair sets: every pair class in sorted order
        used = sorted({q["ky"] for q in self.qcs})
        hs = R.pairsets_multi([self.pcs[y]["pairs"][self.pcs[y]["order"]] for y in used], screen,
                              threads)
        self.khandle = dict(zip(used, hs))
        bh, kh, kc, cls = [], [], [], []
        for k, q in enumerate(self.qcs):
            rows = q["rows"][offset % stride::stride]
            q["sample"] = rows
            bra = self.pcs[q["bx"]]["pairs"]
            for ip, cnt in rows:
                bh.append(tuple(bra[ip]))
                kh.append(self.khandle[q["ky"]])
                kc.append(cnt)
                cls.append(k)
        # the pair lists behind the handles, to build the same rows with
        # another library (mirror)
        self.screen = screen
        self.ket_lists = [self.pcs[y]["pairs"][self.pcs[y]["order"]] for y in used]
        self.ket_index = {y: i for i, y in enumerate(used)}
        self.bra_pairs = bh
        self.bh = R.pairsets_single(bh, screen, threads) if bh else np.zeros(0, np.int32)
        self.kh = np.array(kh, np.int32)
        self.kc = np.array(kc, np.int32)
        self.cls = np.array(cls, np.int32)
        self.setup_s = time.time() - t0
        self.nquartets = int(self.kc.sum()) if len(self.kc) else 0

    def run(self, threads=None, deriv=0, idx=None, count=False):
        """Time the sampled rows (or rows idx): (seconds, primq[] or None)."""
        sel = slice(None) if idx is None else idx
        t, ret, prq = self.R.rows(self.bh[sel], self.kh[sel], self.kc[sel], deriv, self.tol,
                                  threads, count=count)
        return t, prq

    def mirror(self, D, shells, threads=None):
        """The same rows built by library D (a RefLib over another build of
        the simint API): D's own pair sets over the same pair lists.
        Returns (bh, kh, kc) handles of D."""
        D.set_shells(shells)
        hs = D.pairsets_multi(self.ket_lists, self.screen, threads)
        kh = np.array([hs[self.ket_index[self.qcs[k]["ky"]]] for k in self.cls], np.int32)
        bh = D.pairsets_single(self.bra_pairs, self.screen, threads) if self.bra_pairs else \
            np.zeros(0, np.int32)
        return bh, kh, self.kc.copy()

    def layout(self, deriv=0):
        """Offset (doubles) of every sampled row's output and the total."""
        nout = np.array([np.prod([ncart(x) for x in self.qcs[k]["am"]]) for k in self.cls],
                        dtype=np.int64) * (12 if deriv else 1)
        sizes = self.kc.astype(np.int64) * nout
        off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if len(sizes) else \
            np.zeros(0, np.int64)
        return off, int(sizes.sum()) if len(sizes) else 0

    def outputs(self, threads=None, deriv=0):
        """Integrals of every sampled row: (values, offset of each row)."""
        off, n = self.layout(deriv)
        out = np.zeros(n)
        self.R.rows(self.bh, self.kh, self.kc, deriv, self.tol, threads, out=out, off=off,
                    count=False)
        if deriv == 0:
            self.row_off = off
        return out, off

    def class_keys(self, k, nshell):
        """Sorted quartet keys ((i N + j) N + k) N + l of class k's sampled
        rows and the offset (doubles) of each quartet in outputs()."""
        q = self.qcs[k]
        X, Y = self.pcs[q["bx"]], self.pcs[q["ky"]]
        nout = int(np.prod([ncart(x) for x in q["am"]]))
        rows_of_class = np.nonzero(self.cls == k)[0]   # row_off is set by outputs()
        keys, offs = [], []
        for r_local, r in enumerate(rows_of_class):
            ip, cnt = q["sample"][r_local]
            i, j = X["pairs"][ip]
            kl = Y["pairs"][Y["order"][:cnt]].astype(np.int64)
            keys.append(((int(i) * nshell + int(j)) * nshell + kl[:, 0]) * nshell + kl[:, 1])
            offs.append(self.row_off[r] + np.arange(cnt, dtype=np.int64) * nout)
        if not keys:
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        keys = np.concatenate(keys)
        offs = np.concatenate(offs)
        o = np.argsort(keys, kind="stable")
        return keys[o], offs[o]


def compare_class(ref_out, ref_keys, ref_offs, dev_vals, sh4, nout, nshell, chunk=20000):
    """Element-wise comparison of one class of a sweep's output (dev_vals:
    quartet-major, nout doubles per quartet; sh4: shells of each quartet)
    with the reference's values of the same quartets.  Quartets the
    reference rows do not hold (a different cut at the screening boundary)
    are skipped.  Returns (max abs, max rel over |ref| > 1e-15, number
    compared, number of elements beyond the bar: abs > 1e-13 and rel >
    1e-11, number of quartets holding such an element)."""
    sh = sh4.astype(np.int64)
    keys = ((sh[:, 0] * nshell + sh[:, 1]) * nshell + sh[:, 2]) * nshell + sh[:, 3]
    pos = np.searchsorted(ref_keys, keys)
    pos = np.minimum(pos, max(len(ref_keys) - 1, 0))
    hit = (len(ref_keys) > 0) & (ref_keys[pos] == keys) if len(ref_keys) else np.zeros(len(keys), bool)
    qidx = np.nonzero(hit)[0]
    mabs = mrel = 0.0
    nbad = nbadq = 0
    cols = np.arange(nout, dtype=np.int64)
    for c0 in range(0, len(qidx), chunk):
        q = qidx[c0:c0 + chunk]
        g = dev_vals.reshape(-1, nout)[q]
        r = ref_out[ref_offs[pos[q]][:, None] + cols[None, :]]
        d = np.abs(g - r)
        ar = np.abs(r)
        big = ar > 1e-15
        rel = np.where(big, d / np.where(big, ar, 1.0), 0.0)
        mabs = max(mabs, float(d.max()) if d.size else 0.0)
        mrel = max(mrel, float(rel.max()) if rel.size else 0.0)
        beyond = (d > 1e-13) & ((~big) | (rel > 1e-11))
        nbad += int(np.count_nonzero(beyond))
        nbadq += int(np.count_nonzero(beyond.any(axis=1)))
    return mabs, mrel, len(qidx), nbad, nbadq
