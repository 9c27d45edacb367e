#!/usr/bin/env python3
"""Benchmark of the B200 Simint engine (one JSON line on stdout).

Workload ("cfg2"): 500 seeded synthetic shells, s:p:d:f = 200:150:100:50,
1-8 primitives, exponents log-uniform in [0.05, 5e4], 120 pseudo-atoms in a
20 bohr cube; every shell quartet surviving the shell-pair Schwarz test
Q_ab*Q_cd >= 1e-14, primitive screening at the same tolerance, GAMESS
Cartesian ordering.  The full sweep (1.9e9 quartets, 1e11 primitive
quartets) is far beyond one step, so a step is one pass over a proportional
stratified subsample of it: every `--stride`-th bra-pair row of every AM
class (the class mix of the whole sweep is kept).  Metric: evaluated
primitive quartets per second.  `value` is the mixed-precision batched path
(FP32 VRR for primitive quartets whose estimated FP32 error is below
gate / (primitive quartets of their shell quartet), FP64 elsewhere); the
FP64 path is reported beside it.  Both are compared element by element with
the reference's own generated CPU library on the same quartets (max abs and
rel error per class).

Arms:
  default            B200 sweep (device-resident inputs; CUDA-graph replay),
                     plus e2e through simint_compute_eri with host buffers and
                     the reference CPU library timed on the host cores over the
                     same rows (cpu_baseline).
  --impl reference   the reference's generated CPU library (create.py output,
                     all-inline GAMESS build, gcc -O3, OpenMP over rows, all
                     host cores) over the same sampled rows as simint_compute_eri
                     calls (one bra pair x its surviving kets); it loads no
                     part of the B200 library.

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

TOL = 1e-14
MAX_AM = 3
SEED = 2024
GAMESS = 1
REF_VARIANT = "gamess_l3"       # all-inline GAMESS build, max_am 3
LINE_LIMIT = 3000               # bytes of the printed result line (kept well under 4 KB)


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--stride", type=int, default=2000,
                    help="keep every stride-th bra-pair row of each class")
    ap.add_argument("--e2e-stride", type=int, default=40000)
    ap.add_argument("--gate", type=float, default=1e-10,
                    help="mixed precision: bound on the FP32 error of one integral "
                         "(simint_b200_set_precision)")
    ap.add_argument("--cpu-passes", type=int, default=3,
                    help="timed passes of the reference CPU library for cpu_baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the element-wise comparison with the reference library")
    ap.add_argument("--detail", default=None,
                    help="write the per-class table (JSON) to this file")
    return ap.parse_args(argv)


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


METRIC = "primitive quartets/s (cfg2 l<=3 screened sweep sample, screen_tol 1e-14)"


def workload_config(args, world=1):
    """The workload description both arms print."""
    return {"workload": "cfg2 sweep sample: 500 shells s:p:d:f 200:150:100:50, 1-8 prims, "
                        "alpha 0.05-5e4, 120 atoms in 20 bohr, Schwarz 1e-14, GAMESS order; "
                        "every %d-th bra row of every class per rank" % args.stride,
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


def load_reference():
    """(reflib module, refsweep module, RefLib) of the reference's generated
    CPU library, or a reason string when it is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reflib
    import refsweep
    if not reflib.available(REF_VARIANT):
        return None, None, "reference library %s not built (oracle/build_reflib.py)" % (
            os.path.basename(reflib.lib_path(REF_VARIANT)))
    return reflib, refsweep, reflib.load(REF_VARIANT)


def workload_shells(lib):
    from simint_b200.capi import ShellSet
    from simint_b200.workloads import config_shells
    shells = config_shells("cfg2")
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    return shells, S


def pack_bytes(P):
    """Bytes simint_compute_eri uploads for one pair set (packed records)."""
    from simint_b200.capi import padded_nprim
    a256 = lambda n: (n + 255) & ~255
    return a256(padded_nprim(P) * 16 * 8 + 2 * a256(P.nshell12 * 4) + 24 * P.nshell12)


def e2e_rows(sb, lib, S, B, stride, rank=0):
    """Host pair objects (P = one bra pair, Q = its screened ket list) for a
    proportional sample of the sweep's rows."""
    rows = []
    for k, c in enumerate(B.classes()):
        rr = B.rows(k)
        sh4 = B.class_quartets(k, c["nquart"])
        for r in range(rank % stride, len(rr), stride):
            first, n = rr[r]
            P = sb.make_pairs(lib, S, [tuple(sh4[first, :2])], sb.SIMINT_SCREEN_SCHWARZ)
            Q = sb.make_pairs(lib, S, [tuple(x) for x in sh4[first:first + n, 2:]],
                              sb.SIMINT_SCREEN_SCHWARZ)
            rows.append((c["am"], P, Q))
    return rows


def flops_of_class(am, nprimq, nquart):
    from simint_b200.perfmodel import class_flops
    return class_flops(am, nprimq, nquart)


def amname(am):
    return "".join("spdfg"[x] for x in am)


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------

def reference_rate(S, warmup, steps, threads):
    """(primitive quartets/s, seconds per pass, primitive quartets per pass,
    per-pass seconds) of the reference library over the sampled rows."""
    _, prq = S.run(threads, count=True)
    npq = int(prq.sum())
    for _ in range(warmup):
        S.run(threads)
    ts = [S.run(threads)[0] for _ in range(steps)]
    t = sum(ts) / len(ts)
    return npq / t, t, npq, ts


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return          # the CPU reference runs once, on rank 0
    reflib, refsweep, R = load_reference()
    if reflib is None:
        print(json.dumps({"impl": "reference", "unavailable": R}))
        return
    shells = refsweep.workloads().config_shells("cfg2")
    threads = os.cpu_count() or 1
    S = refsweep.RefSweep(R, shells, TOL, MAX_AM, stride=args.stride, offset=0, threads=threads)
    rate, t, npq, _ = reference_rate(S, args.warmup, args.steps, threads)
    sample = ("%d rows (%d shell quartets, %.3g primitive quartets) of the cfg2 sweep sample, "
              "reference %s build (create.py output, gcc -O3, OpenMP over rows)"
              % (len(S.bh), S.nquartets, npq, REF_VARIANT))
    out = {
        "impl": "reference", "metric": METRIC,
        "value": rate, "unit": "primitive quartets/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cfg2 shells, PCG64 seed 2024)",
        "config": dict(workload_config(args), rows=len(S.bh), l2="n/a (CPU)", setup_s=round(S.setup_s, 1),
                       timed="simint_compute_eri per row (one bra pair x its surviving kets)"),
        "cpu_baseline": {"value": rate, "unit": "primitive quartets/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": "primitive quartets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(compact(out))


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


def run_b200(args):
    import torch
    import simint_b200 as sb
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
    lib.simint_b200_set_ordering(GAMESS)
    shells, S = workload_shells(lib)
    t0 = time.time()
    B = sb.Basis(S, TOL, MAX_AM, lib)
    nfull = sum(B.class_full(k) for k in range(len(B.classes())))
    from simint_b200.shard import check_world
    check_world(world, args.stride)
    B.subsample_stride(args.stride, rank)
    npq = B.count_primq()
    classes = B.classes()
    setup_s = time.time() - t0
    stream = torch.cuda.current_stream()
    cap = max(1, min(B.output_size, (4 << 30) // 8))
    out = torch.empty(cap, dtype=torch.float64, device="cuda")
    flush = torch.empty((256 << 20) // 4, dtype=torch.float32, device="cuda")   # > L2 (126 MB)
    peak64 = sb.fma_peak(False, lib)
    peak32 = sb.fma_peak(True, lib)
    gate = args.gate
    # autotune kernel variants per class on this sweep (untimed)
    t1 = time.time()
    for prec in (sb.FP64, sb.MIXED):
        lib.simint_b200_set_precision(prec, gate)
        B.autotune(prec, out.data_ptr(), cap, stream.cuda_stream)
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    tune_s = time.time() - t1

    def timed(prec):
        lib.simint_b200_set_precision(prec, gate)
        nl = 0
        for _ in range(args.warmup):
            nl = B.compute(prec, out.data_ptr(), cap, stream.cuda_stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms = []
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
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        tot = sum(a.elapsed_time(b) for a, b in ms)
        if dist:
            from simint_b200.shard import reduce_time_max
            tot = reduce_time_max(dist, tot, "cuda")
        return tot / args.steps, nl, clk.summary()

    ms64, nl64, clk64 = timed(sb.FP64)
    sums64 = B.checksums()
    msmx, nlmx, clkmx = timed(sb.MIXED)
    sumsmx = B.checksums()
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    ct64 = B.class_times(sb.FP64, out.data_ptr(), cap, stream.cuda_stream)
    full = B.output_size <= cap
    host64 = out[:B.output_size].cpu().numpy() if (full and rank == 0) else None
    lib.simint_b200_set_precision(sb.MIXED, gate)
    ctmx = B.class_times(sb.MIXED, out.data_ptr(), cap, stream.cuda_stream)
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    torch.cuda.synchronize()
    hostmx = out[:B.output_size].cpu().numpy() if (full and rank == 0) else None

    total_npq = npq
    if dist:
        from simint_b200.shard import reduce_count_sum
        total_npq = reduce_count_sum(dist, npq, "cuda")
    value = total_npq / (msmx / 1e3)
    value64 = total_npq / (ms64 / 1e3)

    dom = max(range(len(classes)), key=lambda k: ctmx[k])
    dc = classes[dom]
    dom_fl = flops_of_class(dc["am"], dc["nprimq"], dc["nquart"])
    achieved = dom_fl / (ctmx[dom] / 1e3) / 1e12
    # DRAM bytes of the dominant class's launch: bytes per shell quartet from
    # one ncu capture of that kernel (profiles/traffic.json) times the
    # quartets this launch processes (traffic grows with the output)
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        ent = json.load(open(prof)).get(amname(dc["am"]))
        if ent:
            traffic = ent["dram_bytes_per_quartet"] * dc["nquart"]

    e2e = cpu = check = None
    per_check = [{} for _ in classes]
    if rank == 0:
        # e2e through the reference-facing C ABI, host buffers
        rows = e2e_rows(sb, lib, S, B, max(1, args.e2e_stride // args.stride))
        lib.simint_b200_set_precision(sb.MIXED, gate)
        npq_e2e = sum(sb.count_primq(P, Q, TOL, lib) for _, P, Q in rows)
        h2d = sum(pack_bytes(P) + pack_bytes(Q) for _, P, Q in rows)
        bufs = [np.empty(P.nshell12_clip * Q.nshell12_clip * sb.ncart(P.am1) * sb.ncart(P.am2)
                         * sb.ncart(Q.am1) * sb.ncart(Q.am2)) for _, P, Q in rows]
        d2h = sum(b.nbytes for b in bufs)
        dp = C.POINTER(C.c_double)
        for _ in range(max(1, args.warmup)):
            for (am, P, Q), buf in zip(rows, bufs):
                lib.simint_compute_eri(C.byref(P), C.byref(Q), TOL, None, buf.ctypes.data_as(dp))
        times = []
        for _ in range(args.steps):
            t = time.perf_counter()
            for (am, P, Q), buf in zip(rows, bufs):
                r = lib.simint_compute_eri(C.byref(P), C.byref(Q), TOL, None, buf.ctypes.data_as(dp))
                if r < -1:
                    raise RuntimeError(sb.last_error())
            times.append(time.perf_counter() - t)
        lib.simint_b200_set_precision(sb.FP64, 0.0)
        e2e = {"value": npq_e2e / statistics.median(times), "unit": "primitive quartets/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "calls_per_step": len(rows), "primq_per_step": int(npq_e2e)}
        del bufs, rows
        # the reference's generated CPU library on the host cores, same rows
        reflib, refsweep, R = load_reference() if not (args.no_cpu and args.no_check) else (None, None, "")
        if reflib is not None:
            threads = os.cpu_count() or 1
            RS = refsweep.RefSweep(R, shells, TOL, MAX_AM, stride=args.stride, offset=0,
                                   threads=threads)
            if not args.no_cpu:
                rate, t, n, _ = reference_rate(RS, 1, args.cpu_passes, threads)
                cpu = {"value": rate, "unit": "primitive quartets/s", "cores": threads,
                       "kind": "reference",
                       "sample": "the same %d sampled rows (%.3g primitive quartets, %.2f s per pass, "
                                 "%d passes), reference %s build" % (len(RS.bh), n, t, args.cpu_passes,
                                                                      REF_VARIANT)}
            if not args.no_check and host64 is not None:
                per_check = check_against_reference(B, classes, {"fp64": host64, "mixed": hostmx},
                                                     RS, refsweep, S.n, threads)
                agg = {}
                for name in ("fp64", "mixed"):
                    vals = [e[name] for e in per_check if name in e]
                    agg[name] = {"max_abs": max((v[0] for v in vals), default=None),
                                 "max_rel": max((v[1] for v in vals), default=None),
                                 "quartets": sum(v[2] for v in vals),
                                 "bar_failures": sum(v[3] for v in vals)}
                check = dict(agg, reference=REF_VARIANT,
                             bar="abs <= 1e-13 or rel <= 1e-11 (fp64); mixed: max abs <= gate",
                             gate=gate)
    del host64, hostmx

    per_class = []
    for k, c in enumerate(classes):
        fl = flops_of_class(c["am"], c["nprimq"], c["nquart"])
        ent = {"am": amname(c["am"]), "quartets": c["nquart"], "primq": c["nprimq"],
               "ms_fp64": round(ct64[k], 4), "ms_mixed": round(ctmx[k], 4),
               "primq_s_fp64": c["nprimq"] / max(ct64[k], 1e-9) * 1e3,
               "primq_s_mixed": c["nprimq"] / max(ctmx[k], 1e-9) * 1e3,
               "fp64_tflops": fl / max(ct64[k], 1e-9) / 1e9,
               "checksum_fp64": float(sums64[k, 0]), "checksum_mixed": float(sumsmx[k, 0]),
               "abssum_fp64": float(sums64[k, 1]),
               "variant_fp64": B.variant(c["am"], sb.FP64), "variant_mixed": B.variant(c["am"], sb.MIXED)}
        for name, v in per_check[k].items():
            ent[name + "_vs_ref"] = {"max_abs": v[0], "max_rel": v[1], "quartets": v[2],
                                     "bar_failures": v[3]}
        per_class.append(ent)
    top = sorted(per_class, key=lambda e: -e["ms_mixed"])[:3]

    if rank == 0:
        launches = nlmx // 2 * args.steps      # ERI kernels (checksum kernels excluded)
        res = {
            "metric": METRIC,
            "value": value, "unit": "primitive quartets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": msmx, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32 (FP32 VRR behind the per-integral error gate)",
            "data": "synthetic (seeded cfg2 shells, PCG64 seed 2024)",
            "config": dict(workload_config(args, world), **{
                       "quartets_per_step": int(sum(c["nquart"] for c in classes)),
                       "primq_per_step": int(total_npq), "full_sweep_quartets": int(nfull),
                       "gate": gate, "l2": "256 MB flush before every timed step",
                       "setup_s": round(setup_s, 1), "autotune_s": round(tune_s, 1)}),
            "fp64": {"value": value64, "ms_per_step": ms64},
            "vs_reference_values": check,
            "roofline": {"bound": "fp64", "kernel": "class " + amname(dc["am"]),
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64 if peak64 > 0 else None, "traffic": traffic,
                         "peak_source": "measured FP64 FMA-chain probe, of measured"},
            "top_classes": [{"am": e["am"], "ms": e["ms_mixed"], "tflops": e["fp64_tflops"]} for e in top],
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clkmx,
        }
        if args.detail:
            d = os.path.dirname(os.path.abspath(args.detail))
            os.makedirs(d, exist_ok=True)
            with open(args.detail, "w") as f:
                json.dump(dict(res, per_class=per_class, clocks_fp64=clk64, fp32_peak=peak32), f)
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
