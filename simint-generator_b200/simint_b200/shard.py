"""Sharding of a sweep over ranks (one process per GPU).

Every shell quartet is independent, so ranks split the bra-pair rows of each
AM class with no exchange on the data path: rank r of a job keeps rows
r, r + stride, r + 2 stride, ... of every class (simint_b200_basis_
subsample_stride(b, stride, r)).  Each rank's sample has the class mix and
about the size of a one-rank sample with the same stride (weak scaling); the
samples of different ranks are disjoint while world <= stride.  Results that
need the whole job (primitive-quartet totals, the step time) are reduced on
the host side of torch.distributed: sums for counts, the maximum for times.
"""


def shard_rows(nrows, stride, rank):
    """Rows of one class that rank `rank` sweeps (the same rule as
    simint_b200_basis_subsample_stride with offset = rank)."""
    if stride < 1 or rank < 0:
        raise ValueError("stride >= 1 and rank >= 0 required")
    return list(range(rank % stride, nrows, stride))


def check_world(world, stride):
    """Disjoint shards need world <= stride."""
    if world > stride:
        raise ValueError("world size %d exceeds the row stride %d: shards would overlap" % (world, stride))


def reduce_time_max(dist, ms, device=None):
    """Step time of the job: the slowest rank's device time."""
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_count_sum(dist, n, device=None):
    """Work units of the whole job."""
    import torch
    t = torch.tensor([float(n)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
