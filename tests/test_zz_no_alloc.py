"""GPU: the entry point that allocates nothing (simint_b200_compute_eri_noalloc).

Callers that may not allocate device memory -- a framework that owns the
device memory pool and only hands out buffers, code running while such a
pool is captured, or a hot path that must not hit the implicit
synchronisation of cudaMalloc/cudaFree -- pack their pairs with
simint_b200_pack, copy them into buffers they already own, and call the
allocation-free entry point.  Its results must equal those of the ordinary
simint_compute_eri_deriv on the same pairs, call after call (the shared
static scratch keeps the previous call's contents, which must not leak into
the next result).

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet, PairP
from simint_b200.workloads import random_shells
from oracle import load_oracle
from _util import oracle_pairs, oracle_eri, parity_bad

pytestmark = pytest.mark.gpu


def _bind(lib):
    lib.simint_b200_packed_size.argtypes = [PairP]
    lib.simint_b200_packed_size.restype = C.c_size_t
    lib.simint_b200_pack.argtypes = [PairP, C.c_void_p, C.c_size_t]
    lib.simint_b200_pack.restype = C.c_int
    lib.simint_b200_noalloc_scratch_bytes.restype = C.c_longlong
    lib.simint_b200_compute_eri_noalloc.argtypes = [C.c_int, PairP, C.c_void_p, PairP, C.c_void_p,
                                                   C.c_double, C.c_void_p, C.c_void_p]
    lib.simint_b200_compute_eri_noalloc.restype = C.c_int


def _to_device(torch, lib, P):
    n = lib.simint_b200_packed_size(C.byref(P))
    host = np.zeros((n + 7) // 8, dtype=np.float64)
    assert lib.simint_b200_pack(C.byref(P), host.ctypes.data, host.nbytes) == 0
    return torch.from_numpy(host).cuda()


@pytest.mark.parametrize("am,deriv,screen,tol", [
    ((2, 2, 2, 2), 0, 0, 0.0),       # same (cooperative) kernel on both paths
    ((1, 1, 1, 1), 0, 1, 1e-12),     # straight-line kernel on the ordinary path
    ((2, 1, 0, 1), 1, 0, 0.0),       # first derivatives
], ids=["dddd", "pppp_screened", "dpsp_deriv1"])
def test_noalloc_matches_compute_eri(am, deriv, screen, tol):
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    _bind(lib)
    assert lib.simint_b200_noalloc_scratch_bytes() == 32 * 1024 * 1024
    rng = np.random.default_rng(77 + sum(am) + deriv)
    ams = [am[0]] * 3 + [am[1]] * 2 + [am[2]] * 3 + [am[3]] * 3
    S = ShellSet(random_shells(rng, ams, nprim_range=(1, 3), alpha=(0.1, 30.0), box=4.0))
    lib.simint_normalize_shells(S.n, S.ptr(0))
    bra = [(i, j) for i in (0, 1, 2) for j in (3, 4)]
    ket = [(i, j) for i in (5, 6, 7) for j in (8, 9, 10)]
    P = sb.make_pairs(lib, S, bra, screen)
    Q = sb.make_pairs(lib, S, ket, screen)
    r0, want = sb.compute_eri(P, Q, tol, deriv, lib)
    assert r0 == len(bra) * len(ket)
    # the ordinary entry point against the CPU oracle on the same pairs
    orc = load_oracle()
    oP, oQ = oracle_pairs(orc, S, bra, screen), oracle_pairs(orc, S, ket, screen)
    rr, ref = oracle_eri(orc, oP, oQ, tol, deriv, 0)
    orc.oracle_free_pair(C.byref(oP))
    orc.oracle_free_pair(C.byref(oQ))
    assert rr == r0
    bad, dmax = parity_bad(want, ref)
    assert len(bad) == 0, dmax
    dP, dQ = _to_device(torch, lib, P), _to_device(torch, lib, Q)
    for call in range(2):
        out = torch.full((want.size,), float("nan"), dtype=torch.float64, device="cuda")
        r = lib.simint_b200_compute_eri_noalloc(deriv, C.byref(P), C.c_void_p(dP.data_ptr()),
                                                C.byref(Q), C.c_void_p(dQ.data_ptr()), tol,
                                                C.c_void_p(out.data_ptr()),
                                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert r == r0, (call, r)
        got = out.cpu().numpy()
        bad, dmax = parity_bad(got, want)
        assert len(bad) == 0, (call, dmax)
    lib.simint_free_multi_shellpair(C.byref(P))
    lib.simint_free_multi_shellpair(C.byref(Q))


def test_noalloc_rejects_null_and_unsupported():
    """NULL pair data is SIMINT_B200_ERR_ARG; a class whose shared-memory plan
    exceeds the first cooperative kernel's limit ((gg|gg)) is
    SIMINT_B200_ERR_CLASS, with real device buffers and nothing launched."""
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    _bind(lib)
    assert lib.simint_b200_packed_size(None) == 0
    rng = np.random.default_rng(5)
    S = ShellSet(random_shells(rng, [4, 4, 4, 4], nprim_range=(1, 2), alpha=(0.3, 5.0), box=3.0))
    lib.simint_normalize_shells(S.n, S.ptr(0))
    P = sb.make_pairs(lib, S, [(0, 1)], 0)
    Q = sb.make_pairs(lib, S, [(2, 3)], 0)
    try:
        dP, dQ = _to_device(torch, lib, P), _to_device(torch, lib, Q)
        out = torch.zeros(15 ** 4, dtype=torch.float64, device="cuda")
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        r = lib.simint_b200_compute_eri_noalloc(0, None, C.c_void_p(dP.data_ptr()), C.byref(Q),
                                                C.c_void_p(dQ.data_ptr()), 0.0, C.c_void_p(out.data_ptr()),
                                                stream)
        assert r == -5
        r = lib.simint_b200_compute_eri_noalloc(0, C.byref(P), C.c_void_p(dP.data_ptr()), C.byref(Q),
                                                C.c_void_p(dQ.data_ptr()), 0.0, C.c_void_p(out.data_ptr()),
                                                stream)
        assert r == -3
        torch.cuda.synchronize()
        host = np.zeros(8)
        assert lib.simint_b200_pack(None, host.ctypes.data, host.nbytes) == -5
    finally:
        lib.simint_free_multi_shellpair(C.byref(P))
        lib.simint_free_multi_shellpair(C.byref(Q))
