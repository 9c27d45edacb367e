"""Algorithmic work model of one AM class (the roofline numerator).

FLOPs count FMA as 2 and follow the minimal recurrence plan of gen/plan.py
(the (quartet, m) set the VRR really needs; the reference generator computes
every Cartesian of a class up to its maximum m, OSTEI_VRR_Algorithm_Base.cpp,
so its counts are >= these).  Per primitive quartet: set-up (P-Q distance,
exponent ratios, PA/PB/QC/QD/WP/WQ terms), Boys function (Taylor grid
polynomial per order, or the asymptotic branch plus the downward
recursion), VRR steps, contraction adds into the top elements, three
divisions and one square root counted as one FLOP each.  Per shell quartet:
the HRR transform.
"""

from .gen.emit import unique_class
from .gen.plan import class_plan


def class_flops(am, nprimq, nquart):
    """FP64-equivalent algorithmic FLOPs of nquart shell quartets of class
    `am` (deriv 0) that evaluate nprimq primitive quartets."""
    u = unique_class(am)[0]
    p = class_plan(*u)
    L = p.L
    boys = 16 * (L + 1) if L < 4 else 16 + 3 * L + 20
    setup = 30 + (L + 1)
    per_prim = setup + boys + p.vrr_flops() + p.ntop() + 4
    return nprimq * per_prim + nquart * p.hrr_flops()
