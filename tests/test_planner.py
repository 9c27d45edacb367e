"""The recurrence planner reproduces the reference generator's plan.

Pinned against the generator's own "WORK SIZE" log values (batched
contracted elements, primitive VRR elements, HRR intermediates) and its HRR
flop counts, as logged when generating the reference library."""
import pytest

from simint_b200.gen.plan import class_plan, stepdir
from simint_b200.gen.ordering import psi4_order, gamess_order, psi4_to_gamess_perm

WORK = {  # class: (bcont, prim, cont) as logged by ostei_generator
    (0, 0, 0, 0): (1, 1, 0),
    (1, 1, 1, 1): (81, 149, 81),
    (2, 1, 2, 1): (256, 663, 288),
    (2, 2, 2, 2): (961, 2405, 4332),
    (3, 3, 3, 3): (5476, 17273, 57512),
}
WORK_D1 = {(1, 1, 1, 1): (522, 495, 1323), (2, 2, 2, 2): (5386, 5801, 37116)}
HRR_FLOPS = {(1, 1, 0, 0): 18, (1, 1, 1, 0): 54, (1, 1, 1, 1): 324, (2, 1, 1, 1): 648,
             (2, 2, 2, 2): 10586, (3, 3, 3, 3): 111012, (2, 1, 2, 0): 216}


@pytest.mark.parametrize("am", sorted(WORK))
def test_work_size_deriv0(am):
    assert class_plan(*am).reference_worksize() == WORK[am]


@pytest.mark.parametrize("am", sorted(WORK_D1))
def test_work_size_deriv1(am):
    assert class_plan(*am, deriv=1).reference_worksize() == WORK_D1[am]


@pytest.mark.parametrize("am", sorted(HRR_FLOPS))
def test_hrr_flops(am):
    assert class_plan(*am).hrr_flops() == HRR_FLOPS[am]


def test_stepdir_rule():
    # smallest non-zero exponent, right-most on ties
    assert stepdir((1, 1, 0)) == 1
    assert stepdir((2, 1, 0)) == 1
    assert stepdir((2, 0, 0)) == 0
    assert stepdir((1, 1, 1)) == 2
    assert stepdir((0, 2, 2)) == 2


def test_orderings():
    assert psi4_order(2) == ((2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2))
    assert gamess_order(2)[:3] == ((2, 0, 0), (0, 2, 0), (0, 0, 2))
    for l in (0, 1, 4, 5):
        assert psi4_order(l) == gamess_order(l)
    assert sorted(psi4_to_gamess_perm(3)) == list(range(10))
