"""The sweep plan of a column pipeline (pcc_sweep_plan; host logic, no device).

The reference's shoot (NewtonSolver.cpp:439-468) unpacks the free data as
U_p, psi_c, f_c blocks of Nnewton/3 entries each (unpackSpectralFields), with
Delta at in0[2 Nnewton/3 + 2], and builds the left boundary state from
(f_c, psi_c, Delta) and the right one from (U_p, Delta).  So a Jacobian
column perturbs the left sweep's input only for psi_c, f_c and Delta entries
and the right sweep's only for U_p and Delta entries; the untouched side
starts from the base shoot's state.  The plan must march exactly the moved
sides, the base sides that other columns take, right sides first; with
shoot_both_sides every column marches both sides.
"""
import numpy as np
import pytest

import pcc


def _moved(nn, col):
    """(left moves, right moves) from the block layout alone."""
    if col == nn:  # the base shoot
        return True, True
    block = col // (nn // 3)  # 0 U_p, 1 psi_c, 2 f_c
    delta = col == 2 * nn // 3 + 2
    return block >= 1 or delta, block == 0 or delta


def _model(ntau, c0, c1, both):
    nn = 3 * ntau // 4
    out = []
    for side in (1, 0):
        need_base = False
        for c in range(c0, c1):
            if both or _moved(nn, c)[side]:
                out.append(2 * c + side)
            else:
                need_base = True
        if need_base and not (c0 <= nn < c1):
            out.append(2 * nn + side)
    return out


@pytest.mark.parametrize("ntau", [128, 256, 512, 1024, 2048])
def test_full_build_plan(ntau):
    nn = 3 * ntau // 4
    plan = pcc.sweep_plan(ntau, 0, nn + 1)
    assert plan.tolist() == _model(ntau, 0, nn + 1, False)
    # U_p columns and Delta and the base on the right, psi_c/f_c/Delta/base on the left
    assert len(plan) == nn + 3
    assert len(set(plan.tolist())) == len(plan)
    right = [s for s in plan if s & 1]
    assert plan[: len(right)].tolist() == right  # right sides first
    both = pcc.sweep_plan(ntau, 0, nn + 1, shoot_both_sides=True)
    assert both.tolist() == [2 * c + 1 for c in range(nn + 1)] + [2 * c for c in range(nn + 1)]
    # the Jacobian alone adds the base sides it takes
    assert pcc.sweep_plan(ntau, 0, nn).tolist() == plan.tolist()
    assert len(pcc.sweep_plan(ntau, 0, nn, shoot_both_sides=True)) == 2 * nn


def test_column_ranges_against_the_block_model():
    rng = np.random.default_rng(5)
    for ntau in (128, 1024):
        nn = 3 * ntau // 4
        edges = [0, nn // 3 - 1, nn // 3, nn // 3 + 1, 2 * nn // 3 + 1, 2 * nn // 3 + 2, 2 * nn // 3 + 3, nn - 1,
                 nn, nn + 1]
        cases = [(a, b) for a in edges for b in edges if a < b]
        cases += [tuple(sorted(rng.choice(nn + 2, 2, replace=False))) for _ in range(50)]
        for c0, c1 in cases:
            for both in (False, True):
                assert pcc.sweep_plan(ntau, c0, c1, both).tolist() == _model(ntau, c0, c1, both), (ntau, c0, c1)


def test_every_column_side_has_a_source():
    """Each column's two final states come from a slot the plan marches."""
    for ntau in (128, 512):
        nn = 3 * ntau // 4
        for c0, c1 in [(0, nn), (0, nn + 1), (nn, nn + 1), (10, 20), (nn // 3 - 2, nn // 3 + 2), (200 % nn, nn)]:
            marched = set(pcc.sweep_plan(ntau, c0, c1).tolist())
            for c in range(c0, c1):
                lm, rm = _moved(nn, c)
                assert (2 * c if lm else 2 * nn) in marched
                assert (2 * c + 1 if rm else 2 * nn + 1) in marched


def test_invalid_ranges():
    with pytest.raises(pcc.PccError):
        pcc.sweep_plan(1024, 5, 5)
    with pytest.raises(pcc.PccError):
        pcc.sweep_plan(1024, 0, 770)
    with pytest.raises(pcc.PccError):
        pcc.sweep_plan(1022, 0, 10)
    L = pcc.load()
    assert L.pcc_sweep_plan(128, 0, 0, 97, None, 0) == 99  # count only
