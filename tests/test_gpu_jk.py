"""GPU: Coulomb and exchange matrices digested from a sweep
(simint_b200_basis_jk) against J and K built from the oracle's full ERI
tensor, J_pq = sum_rs (pq|rs) D_rs and K_pq = sum_rs (pr|qs) D_rs, for a
random symmetric density on an s/p/d basis (unscreened sweep, so every
quartet contributes).  The sweep holds each unordered shell pair and each
unordered pair of pairs once, so this checks the degeneracy bookkeeping as
well as the contraction."""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells
from oracle import load_oracle
from _util import oracle_pairs, oracle_eri, NC

pytestmark = pytest.mark.gpu


# s/p/d: every class on the warp-per-quartet kernel; with f shells the
# classes above 3 072 integrals per quartet ((fd|fd), (ff|fd), (ff|ff)) take
# the block-per-quartet kernel
BASES = {"spd": [0, 1, 2, 0, 1, 2, 0, 1, 2], "spdf": [0, 1, 2, 3, 3, 2]}


@pytest.mark.parametrize("ordering,basis", [(0, "spd"), (1, "spd"), (0, "spdf"), (1, "spdf")])
def test_jk_matches_full_tensor(ordering, basis):
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    lib.simint_b200_set_ordering(ordering)
    orc = load_oracle()
    rng = np.random.default_rng(55)
    ams = BASES[basis]
    shells = random_shells(rng, ams, nprim_range=(1, 3), alpha=(0.2, 20.0), box=4.0, natom=3)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    off = np.cumsum([0] + [NC(a) for a in ams])
    nbf = int(off[-1])
    # full tensor from the oracle, shell quartet by shell quartet
    pairs = {}
    for A in range(S.n):
        for B in range(S.n):
            pairs[(A, B)] = oracle_pairs(orc, S, [(A, B)])
    T = np.zeros((nbf, nbf, nbf, nbf))
    for (A, B), P in pairs.items():
        for (Cc, D), Q in pairs.items():
            _, v = oracle_eri(orc, P, Q, 0.0, 0, ordering)
            T[off[A]:off[A + 1], off[B]:off[B + 1], off[Cc]:off[Cc + 1], off[D]:off[D + 1]] = \
                v.reshape(NC(ams[A]), NC(ams[B]), NC(ams[Cc]), NC(ams[D]))
    for P in pairs.values():
        orc.oracle_free_pair(C.byref(P))
    Dm = rng.uniform(-1, 1, (nbf, nbf))
    Dm = 0.5 * (Dm + Dm.T)
    J_ref = np.einsum("pqrs,rs->pq", T, Dm)
    K_ref = np.einsum("prqs,rs->pq", T, Dm)
    # the sweep and its digestion
    B = sb.Basis(S, 0.0, max_am=max(ams), lib=lib)
    assert B.nbf == nbf
    n = B.output_size
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    B.compute(sb.FP64, out.data_ptr(), n)
    dD = torch.from_numpy(Dm).cuda()
    dJ = torch.empty((nbf, nbf), dtype=torch.float64, device="cuda")
    dK = torch.empty((nbf, nbf), dtype=torch.float64, device="cuda")
    for _ in range(2):           # twice: J and K are cleared by every call
        B.jk(out.data_ptr(), n, dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
    torch.cuda.synchronize()
    J, K = dJ.cpu().numpy(), dK.cpu().numpy()
    # the same digestion chunk by chunk through a small scratch buffer (one
    # to a few quartets of the largest class per chunk), through one split
    # between the four class streams, and through a scratch buffer that
    # holds the whole sweep
    nmax = max(c["nout"] for c in B.classes())
    # (one stream through nmax + 7 doubles; four streams through a quarter
    # of 4 nmax + 64 each; the full layout)
    for cap in (nmax + 7, 4 * nmax + 64, n):
        scratch = torch.empty(cap, dtype=torch.float64, device="cuda")
        dJ2, dK2 = torch.empty_like(dJ), torch.empty_like(dK)
        B.compute_jk(sb.FP64, dD.data_ptr(), dJ2.data_ptr(), dK2.data_ptr(), scratch.data_ptr(), cap)
        torch.cuda.synchronize()
        # (atomic adds in another order: equal to rounding)
        assert np.allclose(dJ2.cpu().numpy(), J, rtol=1e-13, atol=1e-13 * np.abs(J).max())
        assert np.allclose(dK2.cpu().numpy(), K, rtol=1e-13, atol=1e-13 * np.abs(K).max())
    B.close()
    lib.simint_b200_set_ordering(0)
    scale = max(np.abs(J_ref).max(), np.abs(K_ref).max())
    assert np.abs(J - J_ref).max() <= 1e-12 * scale, np.abs(J - J_ref).max()
    assert np.abs(K - K_ref).max() <= 1e-12 * scale, np.abs(K - K_ref).max()
    assert np.allclose(J, J.T) and np.allclose(K, K.T)
