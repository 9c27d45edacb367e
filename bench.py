#!/usr/bin/env python3
"""Benchmark of the B200 Simint engine (one JSON line on stdout).

Workload ("cfg2"): 500 seeded synthetic shells, s:p:d:f = 200:150:100:50,
1-8 primitives, exponents log-uniform in [0.05, 5e4], 120 pseudo-atoms in a
20 bohr cube; every shell quartet surviving the shell-pair Schwarz test
Q_ab*Q_cd >= 1e-14, primitive screening at the same tolerance.  The full
sweep (1.9e9 quartets, 1e11 primitive quartets) is far beyond one step, so a
step is one pass over a proportional stratified subsample of it: every
`--stride`-th bra-pair row of every AM class (the class mix of the whole
sweep is kept).  Metric: evaluated primitive quartets per second.  `value`
is the mixed-precision batched path (FP32 VRR for primitive quartets whose
estimated FP32 error is below the gate, FP64 elsewhere); the FP64 path is
reported beside it, with the mixed path's max absolute and relative
deviation from it per class.

Arms:
  default            B200 sweep (device-resident inputs; CUDA-graph replay),
                     plus e2e through simint_compute_eri with host buffers and
                     the CPU oracle timed on the host cores (cpu_baseline).
  --impl reference   the CPU restatement of the reference algorithm (the
                     oracle; the reference's own kernels exist only as its
                     code generator's output) on the host cores, over the
                     same simint_compute_eri calls as e2e.

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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--stride", type=int, default=2000,
                    help="keep every stride-th bra-pair row of each class")
    ap.add_argument("--e2e-stride", type=int, default=40000)
    ap.add_argument("--gate", type=float, default=1e-8,
                    help="mixed precision: FP32 VRR for primitive quartets whose estimated FP32 "
                         "error is below this (simint_b200_set_precision)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


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
                        "alpha 0.05-5e4, 120 atoms in 20 bohr, Schwarz 1e-14; every %d-th bra "
                        "row of every class per rank (rank r: rows r mod %d)" % (args.stride, args.stride),
            "parallelism": "dp%d (disjoint row shards, no data-path collective)" % world}


def workload_shells(lib):
    from simint_b200.capi import ShellSet
    from simint_b200.workloads import config_shells
    shells = config_shells("cfg2")
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    return S


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
        for r in range(rank % stride, len(rr), stride):
            first, n = rr[r]
            q0 = B.quartet(k, first)
            kets = [B.quartet(k, first + i)[2:] for i in range(n)]
            P = sb.make_pairs(lib, S, [q0[:2]], sb.SIMINT_SCREEN_SCHWARZ)
            Q = sb.make_pairs(lib, S, kets, sb.SIMINT_SCREEN_SCHWARZ)
            rows.append((c["am"], P, Q))
    return rows


def flops_of_class(am, nprimq, nquart):
    from simint_b200.perfmodel import class_flops
    return class_flops(am, nprimq, nquart)


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------

def cpu_bench(rows, budget_s, threads):
    """(primq/s, seconds, primq, nrows) of the oracle over a row sample that
    takes about budget_s on `threads` host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import load_oracle
    from simint_b200.capi import PairP
    orc = load_oracle()

    def run(idx):
        PP = (PairP * len(idx))(*[C.pointer(rows[i][1]) for i in idx])
        QQ = (PairP * len(idx))(*[C.pointer(rows[i][2]) for i in idx])
        npq = C.c_longlong()
        cs = C.c_double()
        t = orc.oracle_bench_rows(len(idx), PP, QQ, TOL, threads, C.byref(npq), C.byref(cs))
        return t, npq.value

    # interleave classes so any prefix keeps the class mix
    idx = list(range(0, len(rows), max(1, len(rows) // 64)))[:64]
    t, n = run(idx)
    scale = budget_s / max(t, 1e-3)
    take = max(1, min(len(rows), int(len(idx) * scale)))
    step = max(1, len(rows) // take)
    idx = list(range(0, len(rows), step))[:take]
    t, n = run(idx)
    return n / t, t, n, len(idx)


def run_reference(args):
    import simint_b200 as sb
    lib = sb.load()
    lib.simint_init()
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    S = workload_shells(lib)
    B = sb.Basis(S, TOL, MAX_AM, lib)
    B.subsample_stride(args.stride, 0)
    rows = e2e_rows(sb, lib, S, B, max(1, args.e2e_stride // args.stride))
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        cpu_bench(rows, args.cpu_seconds / 4, threads)
    for _ in range(args.steps):
        rate, t, n, nr = cpu_bench(rows, args.cpu_seconds, threads)
        vals.append((rate, t, n, nr))
    rate = statistics.median(v[0] for v in vals)
    t = statistics.median(v[1] for v in vals)
    out = {
        "impl": "reference", "metric": METRIC,
        "value": rate, "unit": "primitive quartets/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cfg2 shells)",
        "config": dict(workload_config(args), sample_rows=vals[-1][3], l2="n/a (CPU)",
                       timed="simint_compute_eri-shaped rows (1 bra pair x screened kets) of the sample"),
        "cpu_baseline": {"value": rate, "unit": "primitive quartets/s", "cores": threads,
                         "kind": "port",
                         "sample": "%d simint_compute_eri-shaped rows of the cfg2 sweep sample, %.3g primitive quartets"
                                   % (vals[-1][3], vals[-1][2])},
        "e2e": {"value": rate, "unit": "primitive quartets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


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
    S = workload_shells(lib)
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
        torch.cuda.nvtx.range_push("timed_" + ("mixed" if prec == sb.MIXED else "fp64"))
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

    ms64, nl64, clk64 = timed(sb.FP64)
    sums64 = B.checksums()
    msmx, nlmx, clkmx = timed(sb.MIXED)
    sumsmx = B.checksums()
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    ct64 = B.class_times(sb.FP64, out.data_ptr(), cap, stream.cuda_stream)
    full = B.output_size <= cap
    out64 = out.clone() if full else None
    lib.simint_b200_set_precision(sb.MIXED, gate)
    ctmx = B.class_times(sb.MIXED, out.data_ptr(), cap, stream.cuda_stream)
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    torch.cuda.synchronize()
    # deviation of the mixed path from the FP64 path, per class (full-layout
    # output only); relative error over elements above 1e-10 of the class max
    errs = {}
    if full:
        for k, c in enumerate(classes):
            a, n = c["offset"], c["nquart"] * c["nout"]
            if n == 0:
                continue
            d = (out[a:a + n] - out64[a:a + n]).abs()
            ref = out64[a:a + n].abs()
            big = ref > 1e-10 * float(ref.max())
            errs[k] = (float(d.max()), float((d[big] / ref[big]).max()) if bool(big.any()) else 0.0)
        del out64
    # Fock digestion of the (mixed) sweep output: Coulomb and exchange
    # matrices of a seeded symmetric density (simint_b200_basis_jk)
    jk = None
    if full:
        nbf = B.nbf
        g = torch.Generator(device="cpu").manual_seed(SEED)
        Dm = torch.rand((nbf, nbf), generator=g, dtype=torch.float64) - 0.5
        Dm = (0.5 * (Dm + Dm.T)).cuda()
        Jm = torch.empty_like(Dm)
        Km = torch.empty_like(Dm)
        B.jk(out.data_ptr(), cap, Dm.data_ptr(), Jm.data_ptr(), Km.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        jms = []
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            B.jk(out.data_ptr(), cap, Dm.data_ptr(), Jm.data_ptr(), Km.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            jms.append(e0.elapsed_time(e1))
        jt = statistics.median(jms)
        nq = sum(c["nquart"] for c in classes)
        ob = B.output_size * 8
        hbm = None
        mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(mp):
            hbm = json.load(open(mp)).get("hbm_gbs")
        jk = {"ms": jt, "quartets_s": nq / jt * 1e3, "integrals_gb_s": ob / jt / 1e6, "nbf": nbf,
              "hbm_frac": (ob / jt / 1e6) / hbm if hbm else None,
              "note": "J and K of a seeded symmetric density from the sweep sample's integrals "
                      "(reads every integral once from HBM; fraction of the measured copy bandwidth)"}
        del Dm, Jm, Km
    # one-electron matrices of the same basis (simint_b200_oei_matrix):
    # overlap, kinetic energy and the nuclear attraction of the workload's
    # pseudo-atoms (distinct shell centres) as point charges Z = 6
    oei = None
    if full:
        atoms = np.unique(np.array([[S.arr[i].x, S.arr[i].y, S.arr[i].z] for i in range(S.n)]), axis=0)
        cen = np.concatenate([atoms, np.full((len(atoms), 1), 6.0)], axis=1)
        nbf = B.nbf
        M = torch.empty((nbf, nbf), dtype=torch.float64, device="cuda")
        npp = sum(S.arr[i].nprim * S.arr[j].nprim for i in range(S.n) for j in range(i + 1))
        oei = {"nbf": nbf, "ncentre": len(atoms), "shell_pairs": S.n * (S.n + 1) // 2,
               "primitive_pairs": npp,
               "note": "overlap, kinetic and nuclear-attraction matrices of the basis (every unique "
                       "shell pair, both triangles written); potential over the pseudo-atoms, Z = 6"}
        for kind, name in ((sb.OEI_OVERLAP, "overlap"), (sb.OEI_KINETIC, "kinetic"),
                           (sb.OEI_POTENTIAL, "potential")):
            sb.oei_matrix(kind, S, cen, M.data_ptr(), stream.cuda_stream, lib)
            torch.cuda.synchronize()
            t = []
            for _ in range(3):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sb.oei_matrix(kind, S, cen, M.data_ptr(), stream.cuda_stream, lib)
                e1.record(stream)
                e1.synchronize()
                t.append(e0.elapsed_time(e1))
            oei[name + "_ms"] = statistics.median(t)
        oei["potential_items_s"] = npp * len(atoms) / oei["potential_ms"] * 1e3
        del M
    total_npq = npq
    if dist:
        from simint_b200.shard import reduce_count_sum
        total_npq = reduce_count_sum(dist, npq, "cuda")
    value = total_npq / (msmx / 1e3)
    value64 = total_npq / (ms64 / 1e3)

    per_class = []
    for k, c in enumerate(classes):
        fl = flops_of_class(c["am"], c["nprimq"], c["nquart"])
        per_class.append({"am": "".join("spdfg"[x] for x in c["am"]), "quartets": c["nquart"],
                          "primq": c["nprimq"], "ms_fp64": round(ct64[k], 4), "ms_mixed": round(ctmx[k], 4),
                          "primq_s_fp64": c["nprimq"] / max(ct64[k], 1e-9) * 1e3,
                          "primq_s_mixed": c["nprimq"] / max(ctmx[k], 1e-9) * 1e3,
                          "fp64_tflops": fl / max(ct64[k], 1e-9) / 1e9,
                          "checksum_fp64": float(sums64[k, 0]), "checksum_mixed": float(sumsmx[k, 0]),
                          "abssum_fp64": float(sums64[k, 1]),
                          "variant_fp64": B.variant(c["am"], sb.FP64), "variant_mixed": B.variant(c["am"], sb.MIXED),
                          "mixed_max_abs_err": errs.get(k, (None, None))[0],
                          "mixed_max_rel_err": errs.get(k, (None, None))[1]})
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
        ent = json.load(open(prof)).get("".join("spdfg"[x] for x in dc["am"]))
        if ent:
            traffic = ent["dram_bytes_per_quartet"] * dc["nquart"]

    # e2e through the reference-facing C ABI, host buffers
    e2e = None
    cpu = None
    if rank == 0:
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
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            rate, t, n, nr = cpu_bench(rows, args.cpu_seconds, threads)
            cpu = {"value": rate, "unit": "primitive quartets/s", "cores": threads, "kind": "port",
                   "sample": "%d of the e2e simint_compute_eri rows (%.3g primitive quartets, %.1f s)"
                             % (nr, n, t)}

    if rank == 0:
        launches = nlmx // 2 * args.steps      # ERI kernels (checksum kernels excluded)
        res = {
            "metric": METRIC,
            "value": value, "unit": "primitive quartets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": msmx, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32 (FP32 VRR behind the error-estimate gate)",
            "data": "synthetic (seeded cfg2 shells, PCG64 seed 2024)",
            "config": dict(workload_config(args, world), **{
                       "path": "mixed-precision batched sweep (value); FP64 sweep in fp64",
                       "quartets_per_step": int(sum(c["nquart"] for c in classes)),
                       "primq_per_step": int(total_npq), "full_sweep_quartets": int(nfull),
                       "gate": gate, "l2": "256 MB flush before every timed step",
                       "setup_s": round(setup_s, 1), "autotune_s": round(tune_s, 1)}),
            "fp64": {"value": value64, "ms_per_step": ms64},
            "mixed_vs_fp64": {"max_abs_err": max((e[0] for e in errs.values()), default=None),
                              "max_rel_err": max((e[1] for e in errs.values()), default=None),
                              "bar_abs": 1e-10, "classes_checked": len(errs)},
            "roofline": {"bound": "fp64", "kernel": "class " + "".join("spdfg"[x] for x in dc["am"]),
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64 if peak64 > 0 else None, "traffic": traffic,
                         "peak_source": "measured FP64 FMA-chain probe (simint_b200_fma_peak), of measured",
                         "flop_model": "reference generator op counts per unique class (simint_b200.perfmodel)",
                         "fp32_peak": peak32},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "fock_jk": jk, "one_electron": oei,
            "clocks": clkmx, "clocks_fp64": clk64, "per_class": per_class,
        }
        print(json.dumps(res))
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
