"""Per-AM-class benchmark of the device-resident ERI entry point.

    python -m simint_b200.classbench --am 3,2,2,1 [--prec fp64|mixed|both]
        [--variant V] [--nbra 32] [--nket 1024] [--nprim 1,4] [--reps 10]

Builds one rectangle of shell pairs of the requested class (random shells
with the exponent range of the l<=3 workload, 0.05-5e4, log-uniform; pairs
Schwarz-screened), uploads the packed pairs once, and times
simint_b200_compute_eri_device with CUDA events on its stream (256 MB L2
flush before every timed call).  Prints one JSON line: shell and primitive
quartets per second, algorithmic FP64 TFLOP/s (perfmodel.class_flops), the
kernel variant, and for --prec both the mixed path's max absolute and
relative deviation from the FP64 path.  One launch per call, so a profiler
filtered on the kernel sees exactly the class asked for.
"""

import argparse
import ctypes as C
import json

import numpy as np

from . import load, make_pairs, count_primq, get_variant, set_variant, ncart, last_error
from . import FP64, MIXED, SIMINT_SCREEN_SCHWARZ
from .capi import ShellSet, PairP
from .perfmodel import class_flops
from .workloads import random_shells


def _bind(lib):
    lib.simint_b200_packed_size.argtypes = [PairP]
    lib.simint_b200_packed_size.restype = C.c_size_t
    lib.simint_b200_pack.argtypes = [PairP, C.c_void_p, C.c_size_t]
    lib.simint_b200_compute_eri_device.argtypes = [C.c_int, PairP, C.c_void_p, PairP, C.c_void_p,
                                                   C.c_double, C.c_void_p, C.c_void_p]


def device_pairs(torch, lib, P):
    """Packed pair layout of P in a device tensor (simint_b200_pack)."""
    _bind(lib)
    n = lib.simint_b200_packed_size(C.byref(P))
    host = np.zeros((n + 7) // 8, dtype=np.float64)
    if lib.simint_b200_pack(C.byref(P), host.ctypes.data, host.nbytes) != 0:
        raise RuntimeError("simint_b200_pack failed")
    return torch.from_numpy(host).cuda()


def build_case(lib, am, nbra, nket, nprim, seed, alpha=(0.05, 5e4), box=8.0,
               screen=SIMINT_SCREEN_SCHWARZ):
    """Shells and (by default Schwarz-screened) pair sets for an nbra x nket
    rectangle."""
    rng = np.random.default_rng(seed)
    nA = max(1, int(round(np.sqrt(nbra))))
    nB = max(1, nbra // nA)
    nC = max(1, int(round(np.sqrt(nket))))
    nD = max(1, nket // nC)
    ams = [am[0]] * nA + [am[1]] * nB + [am[2]] * nC + [am[3]] * nD
    S = ShellSet(random_shells(rng, ams, nprim_range=nprim, alpha=alpha, box=box, natom=24))
    lib.simint_normalize_shells(S.n, S.ptr(0))
    o = np.cumsum([0, nA, nB, nC, nD])
    bra = [(i, j) for i in range(o[0], o[1]) for j in range(o[1], o[2])]
    ket = [(i, j) for i in range(o[2], o[3]) for j in range(o[3], o[4])]
    P = make_pairs(lib, S, bra, screen)
    Q = make_pairs(lib, S, ket, screen)
    return S, P, Q


def run(am, prec="fp64", variant=None, nbra=32, nket=1024, nprim=(1, 4), reps=10, warmup=3,
        tol=1e-14, gate=1e-8, deriv=0, seed=7, lib=None, screen=SIMINT_SCREEN_SCHWARZ):
    import torch
    lib = lib or load()
    lib.simint_init()
    _bind(lib)
    S, P, Q = build_case(lib, am, nbra, nket, nprim, seed, screen=screen)
    if not screen:
        tol = 0.0
    dP, dQ = device_pairs(torch, lib, P), device_pairs(torch, lib, Q)
    nout = ncart(am[0]) * ncart(am[1]) * ncart(am[2]) * ncart(am[3]) * (12 if deriv else 1)
    nquart = P.nshell12_clip * Q.nshell12_clip
    npq = count_primq(P, Q, tol, lib)
    stream = torch.cuda.Stream()
    flush = torch.empty((256 << 20) // 4, dtype=torch.float32, device="cuda")
    precs = {"fp64": [FP64], "mixed": [MIXED], "both": [FP64, MIXED]}[prec]
    res = {"am": "".join("spdfg"[x] for x in am), "deriv": deriv, "quartets": nquart, "primq": npq,
           "nbra": P.nshell12_clip, "nket": Q.nshell12_clip}
    outs = {}
    for pr in precs:
        if variant is not None and set_variant(am, variant, deriv, pr, lib) != 0:
            raise RuntimeError("variant %d not available: %s" % (variant, last_error()))
        lib.simint_b200_set_precision(pr, gate if pr == MIXED else 0.0)
        out = torch.empty(max(1, nquart * nout), dtype=torch.float64, device="cuda")

        def call():
            r = lib.simint_b200_compute_eri_device(deriv, C.byref(P), C.c_void_p(dP.data_ptr()),
                                                   C.byref(Q), C.c_void_p(dQ.data_ptr()), tol,
                                                   C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
            if r < -1:
                raise RuntimeError("simint_b200_compute_eri_device: " + last_error())

        with torch.cuda.stream(stream):
            for _ in range(warmup):
                call()
            stream.synchronize()
            ms = []
            for _ in range(reps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                call()
                e1.record(stream)
                ms.append((e0, e1))
            stream.synchronize()
        t = float(np.median([a.elapsed_time(b) for a, b in ms]))
        key = "fp64" if pr == FP64 else "mixed"
        res[key] = {"ms": t, "quartets_s": nquart / t * 1e3, "primq_s": npq / t * 1e3,
                    "variant": get_variant(am, deriv, pr, lib)}
        if deriv == 0:
            res[key]["fp64_tflops"] = class_flops(am, npq, nquart) / t / 1e9
        outs[key] = out
        if variant is not None:
            set_variant(am, 0, deriv, pr, lib)
    lib.simint_b200_set_precision(FP64, 0.0)
    if "fp64" in outs and "mixed" in outs:
        d = (outs["mixed"] - outs["fp64"]).abs()
        ref = outs["fp64"].abs()
        res["mixed_max_abs_err"] = float(d.max())
        big = ref > 1e-10
        res["mixed_max_rel_err"] = float((d[big] / ref[big]).max()) if bool(big.any()) else 0.0
        res["max_abs_value"] = float(ref.max())
    lib.simint_free_multi_shellpair(C.byref(P))
    lib.simint_free_multi_shellpair(C.byref(Q))
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--am", required=True, help="a,b,c,d")
    ap.add_argument("--prec", default="fp64", choices=["fp64", "mixed", "both"])
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--deriv", type=int, default=0)
    ap.add_argument("--nbra", type=int, default=32)
    ap.add_argument("--nket", type=int, default=1024)
    ap.add_argument("--nprim", default="1,4")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--gate", type=float, default=1e-8)
    ap.add_argument("--no-screen", action="store_true", help="pairs without Schwarz values, tolerance 0")
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()
    am = tuple(int(x) for x in a.am.split(","))
    nprim = tuple(int(x) for x in a.nprim.split(","))
    print(json.dumps(run(am, a.prec, a.variant, a.nbra, a.nket, nprim, a.reps, a.warmup,
                         gate=a.gate, deriv=a.deriv, seed=a.seed,
                         screen=0 if a.no_screen else SIMINT_SCREEN_SCHWARZ)))


if __name__ == "__main__":
    main()
