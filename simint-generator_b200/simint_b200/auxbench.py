"""Micro-benchmarks of the integral consumers next to the ERI sweep.

    python -m simint_b200.auxbench jk  [--stride 8000] [--reps 5] [--scratch-mb 48]
    python -m simint_b200.auxbench oei [--every 3] [--ncentre 30] [--reps 5]

jk:  Coulomb and exchange matrices (simint_b200_basis_jk) of a seeded
     symmetric density from the FP64 sweep of every stride-th bra row of the
     l <= 3 workload basis (500 shells, s:p:d:f 200:150:100:50, 1-8
     primitives, exponents 0.05-5e4, Schwarz 1e-14); beside it the sweep
     alone and the sweep with its digestion through a scratch buffer of
     scratch-mb MB (simint_b200_basis_compute_jk).
oei: overlap, kinetic-energy and nuclear-attraction matrices
     (simint_b200_oei_matrix) of every `every`-th shell of the same basis over
     ncentre seeded point charges (Z = 6) in the basis' 20 bohr box.

Each call is timed with CUDA events on its stream after one warm-up call;
prints one JSON line (milliseconds per call, median of reps).  One launch per
class per call, so a profiler filtered on a kernel name sees the calls'
launches in order.
"""

import argparse
import json
import statistics

import numpy as np

from . import load, Basis, FP64, OEI_OVERLAP, OEI_KINETIC, OEI_POTENTIAL, oei_matrix
from .capi import ShellSet
from .workloads import config_shells

SCREEN_TOL = 1e-14
MAX_AM = 3


def _basis_shells(lib):
    S = ShellSet(config_shells("cfg2"))
    lib.simint_normalize_shells(S.n, S.ptr(0))
    return S


def _time(torch, stream, fn, reps):
    fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.median(ms)


def run_jk(stride=8000, reps=5, scratch_mb=48):
    import torch
    lib = load()
    lib.simint_init()
    S = _basis_shells(lib)
    B = Basis(S, SCREEN_TOL, MAX_AM, lib)
    B.subsample_stride(stride, 0)
    n = B.output_size
    st = torch.cuda.current_stream()
    out = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
    B.compute(FP64, out.data_ptr(), n, st.cuda_stream)
    nbf = B.nbf
    g = torch.Generator(device="cpu").manual_seed(7)
    D = torch.rand((nbf, nbf), generator=g, dtype=torch.float64) - 0.5
    D = (0.5 * (D + D.T)).cuda()
    J, K = torch.empty_like(D), torch.empty_like(D)
    ms = _time(torch, st, lambda: B.jk(out.data_ptr(), n, D.data_ptr(), J.data_ptr(), K.data_ptr(),
                                       st.cuda_stream), reps)
    # the sweep alone, and the sweep with its digestion through an L2-sized
    # scratch buffer (the integrals never leave L2 for HBM)
    ms_sweep = _time(torch, st, lambda: B.compute(FP64, out.data_ptr(), n, st.cuda_stream), reps)
    cap = min(n, scratch_mb * (1 << 20) // 8)
    scratch = torch.empty(max(cap, 1), dtype=torch.float64, device="cuda")
    J2, K2 = torch.empty_like(D), torch.empty_like(D)
    ms_fused = _time(torch, st, lambda: B.compute_jk(FP64, D.data_ptr(), J2.data_ptr(), K2.data_ptr(),
                                                     scratch.data_ptr(), cap, st.cuda_stream), reps)
    torch.cuda.synchronize()
    dj = float((J2 - J).abs().max()) / max(float(J.abs().max()), 1e-300)
    dk = float((K2 - K).abs().max()) / max(float(K.abs().max()), 1e-300)
    return {"what": "jk", "stride": stride, "nbf": nbf, "quartets": B.nquartets,
            "integrals_mb": n * 8 / 1e6, "ms": ms, "integrals_gb_s": n * 8 / ms / 1e6,
            "sweep_ms": ms_sweep, "sweep_plus_jk_ms": ms_sweep + ms,
            "compute_jk_ms": ms_fused, "scratch_mb": cap * 8 / 2 ** 20,
            "compute_jk_vs_jk_rel": max(dj, dk)}


def run_oei(every=3, ncentre=30, reps=5):
    import torch
    lib = load()
    lib.simint_init()
    full = _basis_shells(lib)
    keep = list(range(0, full.n, every))
    S = ShellSet([(full.arr[i].am, (full.arr[i].x, full.arr[i].y, full.arr[i].z),
                   np.ctypeslib.as_array(full.arr[i].alpha, (full.arr[i].nprim,)).copy(),
                   np.ctypeslib.as_array(full.arr[i].coef, (full.arr[i].nprim,)).copy()) for i in keep])
    rng = np.random.default_rng(11)
    cen = np.concatenate([rng.uniform(0.0, 20.0, (ncentre, 3)), np.full((ncentre, 1), 6.0)], axis=1)
    nbf = sum((S.arr[i].am + 1) * (S.arr[i].am + 2) // 2 for i in range(S.n))
    st = torch.cuda.current_stream()
    M = torch.empty((nbf, nbf), dtype=torch.float64, device="cuda")
    res = {"what": "oei", "shells": S.n, "nbf": nbf, "ncentre": ncentre}
    for kind, name in ((OEI_OVERLAP, "overlap"), (OEI_KINETIC, "kinetic"), (OEI_POTENTIAL, "potential")):
        res[name + "_ms"] = _time(torch, st, lambda: oei_matrix(kind, S, cen, M.data_ptr(), st.cuda_stream, lib),
                                  reps)
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("what", choices=["jk", "oei"])
    ap.add_argument("--stride", type=int, default=8000)
    ap.add_argument("--every", type=int, default=3)
    ap.add_argument("--ncentre", type=int, default=30)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--scratch-mb", type=int, default=48)
    a = ap.parse_args()
    if a.what == "jk":
        print(json.dumps(run_jk(a.stride, a.reps, a.scratch_mb)))
    else:
        print(json.dumps(run_oei(a.every, a.ncentre, a.reps)))


if __name__ == "__main__":
    main()
