"""GPU: the mixed-precision path against the FP64 path.

In mixed mode the VRR of a primitive quartet runs in FP32 when its
estimated FP32 error (simint_b200_set_precision) is below the gate; Boys
values, prefactors, the contraction and the HRR stay FP64.  On a basis with
the exponent range of the l<=3 workload (0.05 - 5e4) and gate 1e-12, every
class of the screened sweep must stay within 1e-10 absolute of the FP64
sweep, the FP32 path must actually have run (some results differ from
FP64), and gate 0 must give the FP64 results (within the FP64 parity bar:
the mixed register kernels are separately compiled code).
"""
import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet
from simint_b200.workloads import random_shells

pytestmark = pytest.mark.gpu

ABS_BAR = 1e-10
GATE = 1e-12


@pytest.fixture(scope="module")
def sweep():
    torch = pytest.importorskip("torch")
    lib = sb.load()
    lib.simint_init()
    lib.simint_b200_set_ordering(0)
    rng = np.random.default_rng(99)
    ams = [0] * 12 + [1] * 9 + [2] * 6 + [3] * 4
    shells = random_shells(rng, ams, nprim_range=(1, 6), alpha=(0.05, 5e4), box=9.0, natom=10)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    B = sb.Basis(S, 1e-14, max_am=3, lib=lib)
    B.subsample_stride(3, 0)
    n = B.output_size
    outs = {}
    for name, prec, gate in (("fp64", sb.FP64, 0.0), ("mixed", sb.MIXED, GATE), ("mixed0", sb.MIXED, 0.0)):
        lib.simint_b200_set_precision(prec, gate)
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        B.compute(prec, out.data_ptr(), n)
        torch.cuda.synchronize()
        outs[name] = out.cpu().numpy()
    lib.simint_b200_set_precision(sb.FP64, 0.0)
    return B, outs


def test_mixed_within_bar_every_class(sweep):
    B, outs = sweep
    ndiff = 0
    for c in B.classes():
        sl = slice(c["offset"], c["offset"] + c["nquart"] * c["nout"])
        d = np.abs(outs["mixed"][sl] - outs["fp64"][sl])
        if d.size:
            assert d.max() <= ABS_BAR, (c["am"], d.max())
            ndiff += int((d > 0).sum())
    assert ndiff > 0, "no primitive quartet took the FP32 path"


def test_gate_zero_is_fp64(sweep):
    B, outs = sweep
    d = np.abs(outs["mixed0"] - outs["fp64"])
    assert d.max() <= 1e-13
