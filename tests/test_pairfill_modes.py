"""The pair-fill mode switch (simint_b200_set_pair_fill) on the host: bad
modes are rejected, and without a CUDA device every mode fills on the host,
bit for bit the reference's shell.c.  (With a device the GPU fill is
compared with the host fill in tests/test_gpu_pairfill.py.)"""
import ctypes as C

import numpy as np
import pytest

import simint_b200 as sb
from simint_b200.capi import ShellSet, pair_arrays
from simint_b200.workloads import random_shells


def _has_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_mode_switch_rejects_bad_modes():
    lib = sb.load()
    assert sb.set_pair_fill(7, lib) == -5
    assert sb.set_pair_fill(-1, lib) == -5
    for m in (sb.PAIR_FILL_HOST, sb.PAIR_FILL_GPU, sb.PAIR_FILL_AUTO):
        assert sb.set_pair_fill(m, lib) == 0
        assert sb.get_pair_fill(lib) == m


@pytest.mark.skipif(_has_device(), reason="with a device the GPU fill runs (tests/test_gpu_pairfill.py)")
def test_every_mode_fills_on_the_host_without_a_device():
    lib = sb.load()
    rng = np.random.default_rng(5)
    shells = random_shells(rng, [1] * 40, nprim_range=(4, 6), alpha=(0.1, 100.0), box=8.0)
    S = ShellSet(shells)
    lib.simint_normalize_shells(S.n, S.ptr(0))
    pairs = [(i, j) for i in range(40) for j in range(40)]
    got = []
    try:
        for m in (sb.PAIR_FILL_HOST, sb.PAIR_FILL_GPU, sb.PAIR_FILL_AUTO):
            sb.set_pair_fill(m, lib)
            P = sb.make_pairs(lib, S, pairs, sb.SIMINT_SCREEN_FASTSCHWARZ)
            got.append(pair_arrays(P))
            lib.simint_free_multi_shellpair(C.byref(P))
    finally:
        sb.set_pair_fill(sb.PAIR_FILL_AUTO, lib)
    for g in got[1:]:
        for k, v in got[0].items():
            if isinstance(v, np.ndarray):
                assert np.array_equal(v, g[k]), k
            else:
                assert v == g[k], k
