"""GPU: the device work queue of the CTA-per-quartet kernels (cooperative and
column) and its bounded wait.

A sweep publishes every task of a launch and closes the queue before the
launch, so no CTA ever waits.  simint_b200_basis_queue_probe runs one class
with a queue the host leaves in another state:

* closed with every task published: the same integrals as the sweep;
* open with nothing published: every CTA's wait runs out, the call returns
  SIMINT_B200_ERR_TIMEOUT and the device stays usable;
* open with half the tasks published: those tasks are computed, the waits
  for the rest run out (SIMINT_B200_ERR_TIMEOUT).

The failure is made on the host (a queue nothing completes); no kernel
faults, traps or spins without a limit.
"""
import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells

pytestmark = pytest.mark.gpu

ERR_TIMEOUT = -6
AM = (2, 2, 2, 2)


@pytest.mark.parametrize("variant", [24, sb.VAR_COL[4], sb.VAR_COL_GROUPS],
                         ids=["cooperative", "column", "column_groups"])
def test_queue_probe(variant):
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    rng = np.random.default_rng(31)
    S = ShellSet(random_shells(rng, [2] * 10, nprim_range=(1, 3), alpha=(0.2, 20.0), box=4.0))
    lib.simint_normalize_shells(S.n, S.ptr(0))
    assert sb.set_variant(AM, variant, 0, sb.FP64, lib) == 0
    try:
        B = sb.Basis(S, 1e-12, 2, lib)
        cls = B.classes()
        k = [c["am"] for c in cls].index(AM)
        c = cls[k]
        n = B.output_size
        full = torch.zeros(n, dtype=torch.float64, device="cuda")
        B.compute(sb.FP64, full.data_ptr(), n)
        sums = B.checksums()
        a, m = c["offset"], c["nquart"] * c["nout"]
        want = full[a:a + m].cpu().numpy()
        assert np.isfinite(want).all() and np.abs(want).max() > 0

        out = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
        assert B.queue_probe(k, c["nquart"], True, 1000, out.data_ptr(), m) == c["nquart"]
        assert np.array_equal(out.cpu().numpy(), want)

        # nothing published, queue open: every wait runs out
        assert B.queue_probe(k, 0, False, 20, out.data_ptr(), m) == ERR_TIMEOUT

        # half published, open: that half is computed, then the waits run out
        half = c["nquart"] // 2
        out.fill_(float("nan"))
        assert B.queue_probe(k, half, False, 20, out.data_ptr(), m) == ERR_TIMEOUT
        got = out.cpu().numpy()
        assert np.array_equal(got[:half * c["nout"]], want[:half * c["nout"]])

        # the device and the basis are usable afterwards
        full.zero_()
        B.compute(sb.FP64, full.data_ptr(), n)
        # (checksums are sums of atomic adds: equal up to summation order)
        assert np.allclose(B.checksums(), sums, rtol=1e-12, atol=1e-12)
        assert np.array_equal(full[a:a + m].cpu().numpy(), want)
        B.close()
    finally:
        sb.set_variant(AM, sb.VAR_DEFAULT, 0, sb.FP64, lib)


def test_queue_probe_rejects_non_queue_kernels():
    """A class on a register kernel takes no work from a queue."""
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    rng = np.random.default_rng(32)
    S = ShellSet(random_shells(rng, [0] * 6 + [1] * 4, nprim_range=(1, 3), alpha=(0.2, 20.0), box=4.0))
    lib.simint_normalize_shells(S.n, S.ptr(0))
    am = (1, 1, 1, 1)
    assert sb.set_variant(am, sb.VAR_STRAIGHT, 0, sb.FP64, lib) == 0
    try:
        B = sb.Basis(S, 1e-12, 1, lib)
        cls = B.classes()
        k = [c["am"] for c in cls].index(am)
        m = cls[k]["nquart"] * cls[k]["nout"]
        out = torch.zeros(m, dtype=torch.float64, device="cuda")
        assert B.queue_probe(k, cls[k]["nquart"], True, 10, out.data_ptr(), m) == -5
        B.close()
    finally:
        sb.set_variant(am, sb.VAR_DEFAULT, 0, sb.FP64, lib)
