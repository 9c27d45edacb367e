#!/usr/bin/env python3
"""Benchmark of the B200 Simint engine (one JSON line on stdout).

Workloads (--config; seeded synthetic shells of simint_b200/workloads.py):

  cfg2 (default)  500 shells s:p:d:f = 200:150:100:50, 1-8 primitives,
                  alpha 0.05-5e4, 120 pseudo-atoms in a 20 bohr cube; every
                  shell quartet surviving Q_ab*Q_cd >= 1e-14, primitive
                  screening at the same tolerance, GAMESS order.  The full
                  sweep (1.9e9 quartets) is far beyond one step: a step is a
                  proportional stratified subsample -- every --stride-th
                  bra-pair row of every AM class (the class mix is kept).
                  Headline: the mixed-precision path (FP32 VRR behind the
                  per-integral error gate), FP64 beside it.
  cfg1            64 shells (32 s, 32 p), 3 primitives, alpha 0.1-100, every
                  unique shell quartet (2 164 240) at screen_tol 0, GAMESS
                  order; headline FP64 (the plain configuration).
  cfg3            the cfg1 quartets, headline mixed precision, FP64 beside.
  cfg5            2000 shells s:p:d:f:g, uneven contraction (s,p 4-12, d 2-6,
                  f,g 1-3), alpha 0.02-1e5, 400 atoms in 40 bohr, screen_tol
                  1e-12, Psi4 order, a row sample of the l <= 4 sweep; output
                  streamed through a 0.5 GB device buffer and checksummed per
                  class; headline mixed.
  cfg4            first derivatives: 300 shells s:p:d, 1-6 primitives, a row
                  sample of the l <= 2 sweep at 1e-14 (Psi4 order), each row
                  one simint_b200_compute_eri_device call (a bra pair against
                  its surviving kets); headline FP64 (the derivative path has
                  no FP32 form).

Metric: evaluated primitive quartets per second (after the reference's
primitive screening).  `value` is device time with inputs resident in HBM;
`e2e` the same metric through simint_compute_eri(_deriv) with host buffers
(uploads and downloads inside the timed region), the calls issued from up to
16 host threads at once as the reference arm runs its rows; `cpu_baseline` the
reference's generated CPU library (create.py output, gcc -O3, OpenMP over
rows) on the same rows, timed on this machine's cores.  Sweep outputs are
compared with the reference's values element by element (cfg1/2/3), by
class checksums (cfg5) or row by row (cfg4).

Arms:
  default            the B200 library.
  --impl reference   the reference's generated CPU library over the same
                     rows, as simint_compute_eri(_deriv) calls (one bra pair
                     x its surviving kets); it loads no part of the B200
                     library.

The last stdout line is a compact JSON object; the per-class table goes to
the file named by --detail (not printed).

N > 1 (torchrun): each rank sweeps a disjoint shard of the same size as the
one-rank sample (rows rank, rank + stride, ... of every class: weak
scaling), no collective on the data path; ranks meet at barriers around the
timed region, the max device time is taken and the primitive-quartet counts
are summed.
"""

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "simint-generator_b200"))

SEED = 2024
T_START = time.time()


def note(msg):
    """One progress line on stderr (the result line is the only stdout)."""
    print("[bench +%.1fs] %s" % (time.time() - T_START, msg), file=sys.stderr, flush=True)

PSI4, GAMESS = 0, 1
E2E_THREADS = min(16, os.cpu_count() or 1)   # host threads issuing the e2e calls
LINE_LIMIT = 3000               # bytes of the printed result line (kept well under 4 KB)
METRIC = "primitive quartets/s per AM class, mixed-prec vs FP64 on 1 B200 at ≤1e-10 abs err"

WORKLOADS = {
    "cfg2": dict(shells="cfg2", tol=1e-14, max_am=3, ordering=GAMESS, ref="gamess_l3", stride=2000,
                 headline="mixed", cap_gb=4.0, e2e_every=20, deriv=0,
                 desc="cfg2 l<=3 sweep sample: 500 shells s:p:d:f 200:150:100:50, 1-8 prims, "
                      "alpha 0.05-5e4, 120 atoms in 20 bohr, Schwarz 1e-14, GAMESS order"),
    "cfg1": dict(shells="cfg1", tol=0.0, max_am=1, ordering=GAMESS, ref="gamess_l3", stride=1,
                 headline="fp64", cap_gb=4.0, e2e_every=1, deriv=0,
                 desc="cfg1: 64 shells (32 s, 32 p), 3 prims, alpha 0.1-100, 8 bohr cube; every unique "
                      "shell quartet, screen_tol 0, GAMESS order"),
    "cfg3": dict(shells="cfg1", tol=0.0, max_am=1, ordering=GAMESS, ref="gamess_l3", stride=1,
                 headline="mixed", cap_gb=4.0, e2e_every=1, deriv=0,
                 desc="cfg3: the cfg1 quartets in mixed precision (FP32 VRR behind the gate) beside FP64"),
    "cfg5": dict(shells="cfg5", tol=1e-12, max_am=4, ordering=PSI4, ref="psi4_l4", stride=80000,
                 headline="mixed", cap_gb=0.5, e2e_every=8, deriv=0, tune=False,
                 desc="cfg5 l<=4 uneven sweep sample: 2000 shells s:p:d:f:g, prims s,p 4-12 d 2-6 f,g 1-3, "
                      "alpha 0.02-1e5, 400 atoms in 40 bohr, Schwarz 1e-12, Psi4 order, output streamed"),
    "cfg4": dict(shells="cfg4", tol=1e-14, max_am=2, ordering=PSI4, ref="psi4_d1_l2", stride=97,
                 headline="fp64", cap_gb=4.0, e2e_every=1, deriv=1,
                 desc="cfg4 deriv=1 l<=2 row sample: 300 shells s:p:d 150:100:50, 1-6 prims, alpha 0.1-1e4, "
                      "80 atoms in 16 bohr, Schwarz 1e-14, Psi4 order, 12 gradient components"),
}
REF_VARIANT = WORKLOADS["cfg2"]["ref"]


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="cfg2", choices=sorted(WORKLOADS))
    ap.add_argument("--stride", type=int, default=None,
                    help="keep every stride-th bra-pair row of each class (default: per config)")
    ap.add_argument("--gate", type=float, default=1e-10,
                    help="mixed precision: bound on the FP32 error of one integral "
                         "(simint_b200_set_precision)")
    ap.add_argument("--cpu-passes", type=int, default=3,
                    help="timed passes of the reference CPU library for cpu_baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the comparison with the reference library")
    ap.add_argument("--detail", default=None,
                    help="write the per-class table (JSON) to this file")
    a = ap.parse_args(argv)
    a.w = WORKLOADS[a.config]
    if a.stride is None:
        a.stride = a.w["stride"]
    return a


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def workload_config(args, world=1):
    """The workload description both arms print."""
    w = args.w
    return {"workload": w["desc"] + ("; every %d-th bra row of every class per rank" % args.stride
                                     if args.stride > 1 else "; every row"),
            "config": args.config,
            "parallelism": "dp%d (disjoint row shards, no data-path collective)" % world}


def compact(res):
    """The printed line: floats rounded to 4 significant digits, None-valued
    keys dropped below the top level; raises past LINE_LIMIT bytes."""
    def rnd(v):
        if isinstance(v, float):
            return float("%.4g" % v)
        if isinstance(v, dict):
            return {k: rnd(x) for k, x in v.items() if x is not None}
        if isinstance(v, (list, tuple)):
            return [rnd(x) for x in v]
        return v
    # top-level keys stay even when null (vs_baseline, cpu_baseline, ...)
    line = json.dumps({k: rnd(v) for k, v in res.items()}, separators=(",", ":"))
    if len(line) > LINE_LIMIT:
        raise ValueError("result line too long (%d bytes)" % len(line))
    return line


def load_reference(variant=REF_VARIANT):
    """(reflib module, refsweep module, RefLib) of the reference's generated
    CPU library, or a reason string when it is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reflib
    import refsweep
    if not reflib.available(variant):
        return None, None, "reference library %s not built (oracle/build_reflib.py)" % (
            os.path.basename(reflib.lib_path(variant)))
    return reflib, refsweep, reflib.load(variant)


def workload_shells(lib, args):
    from simint_b200.capi import ShellSet
    from simint_b200.workloads import config_shells
    shells = config_shells(args.w["shells"])
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    return shells, S


def pack_bytes(P):
    """Bytes simint_compute_eri uploads for one pair set (packed records)."""
    from simint_b200.capi import padded_nprim
    a256 = lambda n: (n + 255) & ~255
    return a256(padded_nprim(P) * 16 * 8 + 2 * a256(P.nshell12 * 4) + 24 * P.nshell12)


def sample_rows(sb, lib, S, B, every, screen):
    """Host pair objects (P = one bra pair, Q = its screened ket list, in
    the sweep's order) for every `every`-th row of the basis's current
    sample: [(class index, am, P, Q)], and the shells of each row's quartets
    ((nket, 4) int arrays)."""
    rows, quartets = [], []
    t = 0
    for k, c in enumerate(B.classes()):
        rr = B.rows(k)
        sh4 = B.class_quartets(k, c["nquart"])
        for first, n in rr:
            if t % every == 0:
                P = sb.make_pairs(lib, S, [tuple(sh4[first, :2])], screen)
                Q = sb.make_pairs(lib, S, [tuple(x) for x in sh4[first:first + n, 2:]], screen)
                rows.append((k, c["am"], P, Q))
                quartets.append((first, sh4[first:first + n]))
            t += 1
    return rows, quartets


def e2e_times(sb, fn, calls, costs, steps, warmup, threads):
    """Host seconds of each of `steps` passes over `calls` (argument tuples
    of fn, a C-ABI call through ctypes, which releases the GIL), issued from
    `threads` host threads at once -- the way an OpenMP loop over bra pairs
    calls the reference (skel/test/test_eri.cpp runs its rows in parallel).
    The calls are split once between persistent threads, largest first to
    the least loaded (a static schedule), so each thread keeps its own
    stream and buffers inside the library from pass to pass.  `warmup`
    untimed passes first."""
    import queue
    import threading
    lists = [[] for _ in range(threads)]
    load = [0.0] * threads
    for c, w in sorted(zip(calls, costs), key=lambda x: -x[1]):
        i = min(range(threads), key=lambda t: load[t])
        lists[i].append(c)
        load[i] += w
    go = [queue.Queue() for _ in range(threads)]
    done = queue.Queue()

    def worker(i):
        while go[i].get():
            err = None
            try:
                for a in lists[i]:
                    if fn(*a) < -1:
                        raise RuntimeError(sb.last_error())
            except Exception as e:         # reported by the issuing thread
                err = e
            done.put(err)

    team = [threading.Thread(target=worker, args=(i,), daemon=True) for i in range(threads)]
    for t in team:
        t.start()

    def one_pass():
        for q in go:
            q.put(True)
        errs = [done.get() for _ in range(threads)]
        for e in errs:
            if e is not None:
                raise e

    try:
        for _ in range(max(1, warmup)):
            one_pass()
        times = []
        for _ in range(steps):
            t = time.perf_counter()
            one_pass()
            times.append(time.perf_counter() - t)
    finally:
        for q in go:
            q.put(False)
        for t in team:
            t.join()
    return times


def free_rows(sb, lib, rows):
    for _, _, P, Q in rows:
        lib.simint_free_multi_shellpair(C.byref(P))
        lib.simint_free_multi_shellpair(C.byref(Q))


def flops_of_class(am, nprimq, nquart, deriv=0):
    from simint_b200.perfmodel import class_flops
    return class_flops(am, nprimq, nquart)


def amname(am):
    return "".join("spdfg"[x] for x in am)


def traffic_of(am, nquart):
    """DRAM bytes of a class's launch from one ncu capture of that kernel
    (profiles/traffic.json: bytes per shell quartet) times the quartets this
    launch processes (traffic grows with the output), or None."""
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(prof):
        return None
    ent = json.load(open(prof)).get(amname(am))
    return ent["dram_bytes_per_quartet"] * nquart if ent else None


# ----------------------------------------------------------------------------
# reference arm
# ----------------------------------------------------------------------------

def reference_rate(S, warmup, steps, threads, deriv=0):
    """(primitive quartets/s, seconds per pass, primitive quartets per pass,
    per-pass seconds) of the reference library over the sampled rows."""
    _, prq = S.run(threads, deriv=deriv, count=True)
    npq = int(prq.sum())
    for _ in range(warmup):
        S.run(threads, deriv=deriv)
    ts = [S.run(threads, deriv=deriv)[0] for _ in range(steps)]
    t = sum(ts) / len(ts)
    return npq / t, t, npq, ts


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return          # the CPU reference runs once, on rank 0
    w = args.w
    reflib, refsweep, R = load_reference(w["ref"])
    if reflib is None:
        print(json.dumps({"impl": "reference", "unavailable": R}))
        return
    shells = refsweep.workloads().config_shells(w["shells"])
    threads = os.cpu_count() or 1
    S = refsweep.RefSweep(R, shells, w["tol"], w["max_am"], stride=args.stride, offset=0, threads=threads)
    rate, t, npq, _ = reference_rate(S, args.warmup, args.steps, threads, w["deriv"])
    sample = ("%d rows (%d shell quartets, %.3g primitive quartets) of the %s sample, reference %s build "
              "(create.py output, gcc -O3, OpenMP over rows)"
              % (len(S.bh), S.nquartets, npq, args.config, w["ref"]))
    out = {
        "impl": "reference", "metric": METRIC,
        "value": rate, "unit": "primitive quartets/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded %s shells, PCG64 seed %d)" % (w["shells"], SEED),
        "config": dict(workload_config(args), rows=len(S.bh), l2="n/a (CPU)", setup_s=round(S.setup_s, 1),
                       timed="simint_compute_eri%s per row (one bra pair x its surviving kets)"
                             % ("_deriv(1)" if w["deriv"] else "")),
        "cpu_baseline": {"value": rate, "unit": "primitive quartets/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": "primitive quartets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(compact(out))


# ----------------------------------------------------------------------------
# comparisons with the reference
# ----------------------------------------------------------------------------

def check_against_reference(B, classes, outs, S, refsweep, nshell, threads):
    """Element-wise comparison of the sweep outputs (dict name -> host array
    in the full layout) with the reference's values for the same quartets.
    Returns per class {name: (max abs, max rel, compared, failures)}."""
    ref_out, _ = S.outputs(threads)
    byam = {tuple(q["am"]): k for k, q in enumerate(S.qcs)}
    res = []
    for k, c in enumerate(classes):
        kr = byam.get(tuple(c["am"]))
        ent = {}
        if kr is None or c["nquart"] == 0:
            res.append(ent)
            continue
        keys, offs = S.class_keys(kr, nshell)
        sh4 = B.class_quartets(k, c["nquart"])
        a, n = c["offset"], c["nquart"] * c["nout"]
        for name, arr in outs.items():
            ent[name] = refsweep.compare_class(ref_out, keys, offs, arr[a:a + n], sh4, c["nout"],
                                               nshell)
        res.append(ent)
    return res


def reference_class_sums(S, threads):
    """Per class of the reference rows: (sum, sum of |values|) of the
    integrals, keyed by AM class."""
    out, off = S.outputs(threads)
    sums = {}
    ends = np.concatenate([off[1:], [len(out)]]) if len(off) else off
    for r in range(len(off)):
        am = tuple(S.qcs[S.cls[r]]["am"])
        blk = out[off[r]:ends[r]]
        s = sums.setdefault(am, [0.0, 0.0])
        s[0] += float(blk.sum())
        s[1] += float(np.abs(blk).sum())
    return sums


def aggregate(per_check, names, extra):
    agg = {}
    for name in names:
        vals = [e[name] for e in per_check if name in e]
        agg[name] = {"max_abs": max((v[0] for v in vals), default=None),
                     "max_rel": max((v[1] for v in vals), default=None),
                     "quartets": sum(v[2] for v in vals),
                     "bar_failures": sum(v[3] for v in vals),
                     "bar_failure_quartets": sum(v[4] for v in vals)}
    return dict(agg, **extra)


# ----------------------------------------------------------------------------
# B200 arm: device-resident sweeps (cfg1, cfg2, cfg3, cfg5)
# ----------------------------------------------------------------------------

def run_b200(args):
    import torch
    import simint_b200 as sb
    w = args.w
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    lib = sb.load()
    lib.simint_init()
    lib.simint_b200_set_ordering(w["ordering"])
    shells, S = workload_shells(lib, args)
    if w["deriv"]:
        return run_b200_rows(args, torch, sb, lib, shells, S, rank, world, local, dist)
    tol = w["tol"]
    t0 = time.time()
    B = sb.Basis(S, tol, w["max_am"], lib)
    nfull = sum(B.class_full(k) for k in range(len(B.classes())))
    from simint_b200.shard import check_world
    check_world(world, args.stride)
    if args.stride > 1 or rank > 0:
        B.subsample_stride(args.stride, rank)
    npq = B.count_primq()
    classes = B.classes()
    setup_s = time.time() - t0
    note("basis set up: %d classes, %d primitive quartets, %.1f s" % (len(classes), npq, setup_s))
    stream = torch.cuda.current_stream()
    cap = max(1, min(B.output_size, int(w["cap_gb"] * (1 << 30)) // 8))
    full = B.output_size <= cap
    out = torch.empty(cap, dtype=torch.float64, device="cuda")
    flush = torch.empty((256 << 20) // 4, dtype=torch.float32, device="cuda")   # > L2 (126 MB)
    peak64 = sb.fma_peak(False, lib)
    peak32 = sb.fma_peak(True, lib)
    gate = args.gate
    # autotune kernel variants per class on this sweep (untimed)
    t1 = time.time()
    if w.get("tune", True):
        for prec in (sb.FP64, sb.MIXED):
            lib.simint_b200_set_precision(prec, gate)
            B.autotune(prec, out.data_ptr(), cap, stream.cuda_stream)
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    tune_s = time.time() - t1
    note("autotuned in %.1f s" % tune_s)

    def timed(prec, tag):
        lib.simint_b200_set_precision(prec, gate)
        nl = 0
        for _ in range(args.warmup):
            nl = B.compute(prec, out.data_ptr(), cap, stream.cuda_stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms = []
        torch.cuda.nvtx.range_push(tag)
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                nl = B.compute(prec, out.data_ptr(), cap, stream.cuda_stream)
                e1.record(stream)
                ms.append((e0, e1))
            torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        tot = sum(a.elapsed_time(b) for a, b in ms)
        if dist:
            from simint_b200.shard import reduce_time_max
            tot = reduce_time_max(dist, tot, "cuda")
        return tot / args.steps, nl, clk.summary()

    ms64, nl64, clk64 = timed(sb.FP64, "timed_fp64")
    note("timed FP64: %.3f ms per step" % ms64)
    sums64 = B.checksums()
    msmx, nlmx, clkmx = timed(sb.MIXED, "timed_mixed")
    sumsmx = B.checksums()
    fp32 = B.fp32_counts()
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    # per-class runs, one class after another in class order (the NVTX
    # ranges let a profiler capture exactly these launches)
    torch.cuda.nvtx.range_push("class_times_fp64")
    ct64 = B.class_times(sb.FP64, out.data_ptr(), cap, stream.cuda_stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    host64 = out[:B.output_size].cpu().numpy() if (full and rank == 0) else None
    lib.simint_b200_set_precision(sb.MIXED, gate)
    torch.cuda.nvtx.range_push("class_times_mixed")
    ctmx = B.class_times(sb.MIXED, out.data_ptr(), cap, stream.cuda_stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    torch.cuda.synchronize()
    hostmx = out[:B.output_size].cpu().numpy() if (full and rank == 0) else None

    total_npq = npq
    if dist:
        from simint_b200.shard import reduce_count_sum
        total_npq = reduce_count_sum(dist, npq, "cuda")
    head_mixed = w["headline"] == "mixed"
    ms_head = msmx if head_mixed else ms64
    value = total_npq / (ms_head / 1e3)
    value64 = total_npq / (ms64 / 1e3)
    valuemx = total_npq / (msmx / 1e3)
    ct_head = ctmx if head_mixed else ct64

    dom = max(range(len(classes)), key=lambda k: ct_head[k])
    dc = classes[dom]
    dom_fl = flops_of_class(dc["am"], dc["nprimq"], dc["nquart"])
    achieved = dom_fl / (ct_head[dom] / 1e3) / 1e12
    traffic = traffic_of(dc["am"], dc["nquart"])

    e2e = cpu = check = None
    per_check = [{} for _ in classes]
    if rank == 0:
        # e2e through the reference-facing C ABI, host buffers
        screen = sb.SIMINT_SCREEN_SCHWARZ if tol > 0 else sb.SIMINT_SCREEN_NONE
        rows, rowq = sample_rows(sb, lib, S, B, w["e2e_every"], screen)
        prec_e2e = sb.MIXED if head_mixed else sb.FP64
        lib.simint_b200_set_precision(prec_e2e, gate)
        npq_e2e = sum(sb.count_primq(P, Q, tol, lib) for _, _, P, Q in rows)
        h2d = sum(pack_bytes(P) + pack_bytes(Q) for _, _, P, Q in rows)
        bufs = [np.empty(P.nshell12_clip * Q.nshell12_clip * sb.ncart(P.am1) * sb.ncart(P.am2)
                         * sb.ncart(Q.am1) * sb.ncart(Q.am2)) for _, _, P, Q in rows]
        d2h = sum(b.nbytes for b in bufs)
        dp = C.POINTER(C.c_double)
        calls = [(C.byref(P), C.byref(Q), tol, None, buf.ctypes.data_as(dp)) for (_, am, P, Q), buf in zip(rows, bufs)]
        cost = [b.size + pack_bytes(Q) / 8 for (_, _, P, Q), b in zip(rows, bufs)]
        nthr = max(1, min(len(calls), E2E_THREADS))
        times = e2e_times(sb, lib.simint_compute_eri, calls, cost, args.steps, args.warmup, nthr)
        lib.simint_b200_set_precision(sb.FP64, 0.0)
        note("e2e: %d calls on %d host threads, %.1f ms per step" % (len(rows), nthr, 1e3 * statistics.median(times)))
        e2e = {"value": npq_e2e / statistics.median(times), "unit": "primitive quartets/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "calls_per_step": len(rows), "host_threads": nthr, "primq_per_step": int(npq_e2e),
               "precision": "mixed" if head_mixed else "fp64"}
        # the calls' results against the sweep's values of the same quartets
        # (each call's ket list holds only the row's kets, so the 8-wide
        # vector screening of its last vector may keep or drop a few
        # sub-threshold primitive quartets the sweep's clipped list does not)
        hsw = hostmx if head_mixed else host64
        if hsw is not None:
            dmax = 0.0
            for (k, am, P, Q), buf, (first, q4) in zip(rows, bufs, rowq):
                nout = classes[k]["nout"]
                a0 = classes[k]["offset"] + first * nout
                dmax = max(dmax, float(np.abs(buf - hsw[a0:a0 + buf.size]).max()) if buf.size else 0.0)
            e2e["vs_sweep_max_abs"] = dmax
        del bufs
        free_rows(sb, lib, rows)
        # the reference's generated CPU library on the host cores, same rows
        reflib, refsweep, R = load_reference(w["ref"]) if not (args.no_cpu and args.no_check) \
            else (None, None, "")
        if reflib is not None:
            threads = os.cpu_count() or 1
            RS = refsweep.RefSweep(R, shells, tol, w["max_am"], stride=args.stride, offset=0,
                                   threads=threads)
            if not args.no_cpu:
                rate, t, n, _ = reference_rate(RS, 1, args.cpu_passes, threads)
                note("reference CPU baseline: %.3g primitive quartets/s" % rate)
                cpu = {"value": rate, "unit": "primitive quartets/s", "cores": threads,
                       "kind": "reference",
                       "sample": "the same %d sampled rows (%.3g primitive quartets, %.2f s per pass, "
                                 "%d passes), reference %s build" % (len(RS.bh), n, t, args.cpu_passes,
                                                                      w["ref"])}
            if not args.no_check and full:
                per_check = check_against_reference(B, classes, {"fp64": host64, "mixed": hostmx},
                                                     RS, refsweep, S.n, threads)
                check = aggregate(per_check, ("fp64", "mixed"),
                                  dict(reference=w["ref"], gate=gate,
                                       bar="abs <= 1e-13 or rel <= 1e-11 per element; quartets beyond it are "
                                           "ill-conditioned (tests judge them against a long-double evaluation)"))
            elif not args.no_check:
                # streamed output: class checksums against the reference's
                # sums over the same rows
                rsum = reference_class_sums(RS, threads)
                worst = {"fp64": 0.0, "mixed": 0.0}
                ncls = 0
                for k, c in enumerate(classes):
                    rs = rsum.get(tuple(c["am"]))
                    if rs is None:
                        continue
                    ncls += 1
                    scale = max(rs[1], 1e-300)
                    for name, sums in (("fp64", sums64), ("mixed", sumsmx)):
                        d = abs(float(sums[k, 0]) - rs[0]) / scale
                        per_check[k][name] = (abs(float(sums[k, 0]) - rs[0]), d, c["nquart"], 0, 0)
                        worst[name] = max(worst[name], d)
                check = {"kind": "class checksums vs reference sums over the same rows",
                         "classes": ncls, "fp64_max_rel_sum": worst["fp64"],
                         "mixed_max_rel_sum": worst["mixed"], "reference": w["ref"]}
    del host64, hostmx

    per_class = []
    for k, c in enumerate(classes):
        fl = flops_of_class(c["am"], c["nprimq"], c["nquart"])
        ent = {"am": amname(c["am"]), "quartets": c["nquart"], "primq": c["nprimq"],
               "fp32_primq": int(fp32[k]),
               "ms_fp64": round(ct64[k], 4), "ms_mixed": round(ctmx[k], 4),
               "primq_s_fp64": c["nprimq"] / max(ct64[k], 1e-9) * 1e3,
               "primq_s_mixed": c["nprimq"] / max(ctmx[k], 1e-9) * 1e3,
               "fp64_tflops": fl / max(ct64[k], 1e-9) / 1e9,
               "checksum_fp64": float(sums64[k, 0]), "checksum_mixed": float(sumsmx[k, 0]),
               "abssum_fp64": float(sums64[k, 1]),
               "variant_fp64": B.variant(c["am"], sb.FP64), "variant_mixed": B.variant(c["am"], sb.MIXED)}
        for name, v in per_check[k].items():
            ent[name + "_vs_ref"] = {"max_abs": v[0], "max_rel": v[1], "quartets": v[2],
                                     "bar_failures": v[3], "bar_failure_quartets": v[4]}
        per_class.append(ent)
    top = sorted(per_class, key=lambda e: -(e["ms_mixed"] if head_mixed else e["ms_fp64"]))[:3]
    nfp32 = int(fp32.sum())

    if rank == 0:
        nl_head = nlmx if head_mixed else nl64
        res = {
            "metric": METRIC,
            "value": value, "unit": "primitive quartets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_head, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64+f32 (FP32 VRR behind the per-integral error gate)" if head_mixed else "f64",
            "data": "synthetic (seeded %s shells, PCG64 seed %d)" % (w["shells"], SEED),
            "config": dict(workload_config(args, world), **{
                       "headline": w["headline"],
                       "quartets_per_step": int(sum(c["nquart"] for c in classes)),
                       "primq_per_step": int(total_npq), "full_sweep_quartets": int(nfull),
                       "output": "full layout" if full else "streamed through %.2g GB" % (cap * 8 / 2 ** 30),
                       "gate": gate, "l2": "256 MB flush before every timed step",
                       "setup_s": round(setup_s, 1),
                       "autotune_s": round(tune_s, 1) if w.get("tune", True) else "off (default variant rules)"}),
            "fp64": {"value": value64, "ms_per_step": ms64},
            "mixed": {"value": valuemx, "ms_per_step": msmx, "fp32_primq_frac": nfp32 / max(npq, 1),
                      "classes_with_fp32": int((fp32 > 0).sum()), "classes": len(classes)},
            "vs_reference_values": check,
            "roofline": {"bound": "fp64", "kernel": "class " + amname(dc["am"]),
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64 if peak64 > 0 else None, "traffic": traffic,
                         "peak_source": "measured FP64 FMA-chain probe, of measured"},
            "top_classes": [{"am": e["am"], "ms": e["ms_mixed"] if head_mixed else e["ms_fp64"],
                             "tflops": e["fp64_tflops"]} for e in top],
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": nl_head * args.steps,
            "clocks": clkmx if head_mixed else clk64,
        }
        if args.detail:
            d = os.path.dirname(os.path.abspath(args.detail))
            os.makedirs(d, exist_ok=True)
            with open(args.detail, "w") as f:
                json.dump(dict(res, per_class=per_class, clocks_fp64=clk64, clocks_mixed=clkmx,
                               fp32_peak=peak32), f)
        print(compact(res))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------------------
# B200 arm: first derivatives (cfg4), one device call per row
# ----------------------------------------------------------------------------

def run_b200_rows(args, torch, sb, lib, shells, S, rank, world, local, dist):
    """Rows of the screened l <= 2 sweep (one bra pair against its surviving
    kets), each a simint_b200_compute_eri_device(deriv=1) call on pair data
    already in HBM; all rows of a step back to back on one stream."""
    w = args.w
    tol = w["tol"]
    t0 = time.time()
    B = sb.Basis(S, tol, w["max_am"], lib)
    from simint_b200.shard import check_world
    check_world(world, args.stride)
    B.subsample_stride(args.stride, rank)
    rows, rowq = sample_rows(sb, lib, S, B, 1, sb.SIMINT_SCREEN_SCHWARZ)
    classes = B.classes()
    PairP = C.POINTER(sb.SimintMultiShellpair)
    lib.simint_b200_packed_size.argtypes = [PairP]
    lib.simint_b200_packed_size.restype = C.c_size_t
    lib.simint_b200_pack.argtypes = [PairP, C.c_void_p, C.c_size_t]
    lib.simint_b200_compute_eri_device.argtypes = [C.c_int, PairP, C.c_void_p, PairP, C.c_void_p,
                                                   C.c_double, C.c_void_p, C.c_void_p]
    # pack every row's pairs into one device buffer; outputs into another
    offs, total = [], 0
    for _, _, P, Q in rows:
        a = (lib.simint_b200_packed_size(C.byref(P)) + 255) & ~255
        b = (lib.simint_b200_packed_size(C.byref(Q)) + 255) & ~255
        offs.append((total, total + a))
        total += a + b
    host = np.zeros(total // 8 + 1)
    for (_, _, P, Q), (oa, ob) in zip(rows, offs):
        assert lib.simint_b200_pack(C.byref(P), host.ctypes.data + oa, ob - oa) == 0
        assert lib.simint_b200_pack(C.byref(Q), host.ctypes.data + ob, total - ob) == 0
    dpairs = torch.from_numpy(host).cuda()
    base = dpairs.data_ptr()
    nouts = [P.nshell12_clip * Q.nshell12_clip * sb.ncart(P.am1) * sb.ncart(P.am2) * sb.ncart(Q.am1)
             * sb.ncart(Q.am2) * 12 for _, _, P, Q in rows]
    ooff = np.concatenate([[0], np.cumsum(nouts)]).astype(np.int64)
    dout = torch.zeros(int(ooff[-1]), dtype=torch.float64, device="cuda")
    npq = sum(sb.count_primq(P, Q, tol, lib) for _, _, P, Q in rows)
    setup_s = time.time() - t0
    stream = torch.cuda.current_stream()
    flush = torch.empty((256 << 20) // 4, dtype=torch.float32, device="cuda")
    lib.simint_b200_set_precision(sb.FP64, 0.0)

    def sweep(sel=None):
        for i in (range(len(rows)) if sel is None else sel):
            _, _, P, Q = rows[i]
            oa, ob = offs[i]
            r = lib.simint_b200_compute_eri_device(1, C.byref(P), C.c_void_p(base + oa), C.byref(Q),
                                                   C.c_void_p(base + ob), tol,
                                                   C.c_void_p(dout.data_ptr() + 8 * int(ooff[i])),
                                                   C.c_void_p(stream.cuda_stream))
            if r < -1:
                raise RuntimeError("compute_eri_device: " + sb.last_error())

    for _ in range(args.warmup):
        sweep()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    n0 = lib.simint_b200_launch_count()
    ms = []
    torch.cuda.nvtx.range_push("timed_fp64")
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sweep()
            e1.record(stream)
            ms.append((e0, e1))
        torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    launches = lib.simint_b200_launch_count() - n0
    if dist:
        dist.barrier()
    tot = sum(a.elapsed_time(b) for a, b in ms)
    if dist:
        from simint_b200.shard import reduce_time_max, reduce_count_sum
        tot = reduce_time_max(dist, tot, "cuda")
        npq_all = reduce_count_sum(dist, npq, "cuda")
    else:
        npq_all = npq
    ms_step = tot / args.steps
    value = npq_all / (ms_step / 1e3)
    # per class device time (one untimed pass, events around each class's rows)
    ct = []
    for k, c in enumerate(classes):
        sel = [i for i, r in enumerate(rows) if r[0] == k]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sweep(sel)
        e1.record(stream)
        torch.cuda.synchronize()
        ct.append(e0.elapsed_time(e1))
    calc = dout.cpu().numpy()

    e2e = cpu = check = None
    if rank == 0:
        bufs = [np.empty(n) for n in nouts]
        dp = C.POINTER(C.c_double)
        calls = [(1, C.byref(P), C.byref(Q), tol, None, buf.ctypes.data_as(dp)) for (_, _, P, Q), buf in zip(rows, bufs)]
        cost = [b.size + pack_bytes(Q) / 8 for (_, _, P, Q), b in zip(rows, bufs)]
        nthr = max(1, min(len(calls), E2E_THREADS))
        times = e2e_times(sb, lib.simint_compute_eri_deriv, calls, cost, args.steps, args.warmup, nthr)
        note("e2e: %d calls on %d host threads, %.1f ms per step" % (len(rows), nthr, 1e3 * statistics.median(times)))
        e2e = {"value": npq / statistics.median(times), "unit": "primitive quartets/s",
               "h2d_bytes_per_step": int(sum(pack_bytes(P) + pack_bytes(Q) for _, _, P, Q in rows)),
               "d2h_bytes_per_step": int(sum(b.nbytes for b in bufs)), "calls_per_step": len(rows),
               "host_threads": nthr, "precision": "fp64"}
        reflib, refsweep, R = load_reference(w["ref"]) if not (args.no_cpu and args.no_check) \
            else (None, None, "")
        if reflib is not None:
            threads = os.cpu_count() or 1
            RS = refsweep.RefSweep(R, shells, tol, w["max_am"], stride=args.stride, offset=0, threads=threads)
            if not args.no_cpu:
                rate, t, n, _ = reference_rate(RS, 1, args.cpu_passes, threads, deriv=1)
                note("reference CPU baseline: %.3g primitive quartets/s" % rate)
                cpu = {"value": rate, "unit": "primitive quartets/s", "cores": threads, "kind": "reference",
                       "sample": "the same %d rows (%.3g primitive quartets, %.2f s per pass), reference %s "
                                 "build" % (len(RS.bh), n, t, w["ref"])}
            if not args.no_check:
                ref, roff = RS.outputs(threads, deriv=1)
                # rows matched by (class, bra pair) with identical ket lists
                refrow = {}
                for r in range(len(RS.bh)):
                    q = RS.qcs[RS.cls[r]]
                    refrow[(tuple(q["am"]), tuple(int(x) for x in RS.bra_pairs[r]))] = r
                mabs = mrel = 0.0
                nq = nbad = nskip = 0
                for i, (k, am, P, Q) in enumerate(rows):
                    q4 = rowq[i][1]
                    n = len(q4)
                    key = (tuple(am), tuple(int(x) for x in q4[0, :2]))
                    r = refrow.get(key)
                    if r is None or RS.kc[r] != n:
                        nskip += 1
                        continue
                    y = RS.qcs[RS.cls[r]]
                    kl = RS.pcs[y["ky"]]["pairs"][RS.pcs[y["ky"]]["order"][:n]]
                    if not np.array_equal(kl, q4[:, 2:]):
                        nskip += 1
                        continue
                    g = calc[ooff[i]:ooff[i + 1]]
                    f = ref[roff[r]:roff[r] + nouts[i]]
                    d = np.abs(g - f)
                    big = np.abs(f) > 1e-15
                    rel = np.where(big, d / np.where(big, np.abs(f), 1.0), 0.0)
                    mabs = max(mabs, float(d.max()) if d.size else 0.0)
                    mrel = max(mrel, float(rel.max()) if rel.size else 0.0)
                    nbad += int(np.count_nonzero((d > 1e-13) & ((~big) | (rel > 1e-11))))
                    nq += n
                check = {"fp64": {"max_abs": mabs, "max_rel": mrel, "quartets": nq, "bar_failures": nbad},
                         "rows_skipped": nskip, "reference": w["ref"],
                         "bar": "abs <= 1e-13 or rel <= 1e-11 per gradient element"}
    free_rows(sb, lib, rows)

    dom = max(range(len(classes)), key=lambda k: ct[k])
    dc = classes[dom]
    if rank == 0:
        res = {
            "metric": METRIC,
            "value": value, "unit": "primitive quartets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded %s shells, PCG64 seed %d)" % (w["shells"], SEED),
            "config": dict(workload_config(args, world), **{
                "headline": "fp64 (deriv 1)", "rows_per_step": len(rows), "primq_per_step": int(npq_all),
                "quartets_per_step": int(sum(c["nquart"] for c in classes)),
                "l2": "256 MB flush before every timed step", "setup_s": round(setup_s, 1),
                "timed": "simint_b200_compute_eri_device(1, ...) per row, pair data resident"}),
            "vs_reference_values": check,
            "roofline": {"bound": "fp64", "kernel": "class " + amname(dc["am"]) + " deriv1",
                         "achieved": None, "peak": sb.fma_peak(False, lib), "unit": "TFLOP/s",
                         "traffic": None, "peak_source": "measured FP64 FMA-chain probe, of measured"},
            "top_classes": [{"am": amname(classes[k]["am"]), "ms": ct[k]}
                            for k in sorted(range(len(classes)), key=lambda k: -ct[k])[:3]],
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if args.detail:
            with open(args.detail, "w") as f:
                json.dump(dict(res, per_class=[{"am": amname(c["am"]), "quartets": c["nquart"], "ms": ct[k]}
                                               for k, c in enumerate(classes)]), f)
        print(compact(res))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
