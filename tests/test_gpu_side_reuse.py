"""Side reuse (pcc_solve_desc.shoot_both_sides = 0, the default) against full
two-sided shoots per column (shoot_both_sides = 1, the schedule of the
reference's NewtonSolver::assembleJacobian, NewtonSolver.cpp:615-650).

A column that perturbs a U_p entry leaves the left boundary state bit for bit
the base shoot's, and a psi_c or f_c entry leaves the right one (the left
expansion reads f_c, psi_c and Delta, the right one U_p and Delta:
NewtonSolver.cpp:461-468), so the untouched side's march is the base shoot's
march of the same bits and its final state is taken from there.  Everything
the two schedules return must therefore be identical bit for bit: Jacobians
(single, column ranges across the block edges, batched), the device Newton
loop's iterates, and where a sweep fails, the failing column, side and grid
index.  Only the work differs (about half the sweeps).
"""
import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu


def _pair(engine, cfg, **over):
    import pcc

    c = dict(cfg)
    c.update(over)
    reuse = engine.solve(pcc.SolveDesc.from_config(c))
    both = engine.solve(pcc.SolveDesc.from_config(dict(c, ShootBothSides=True)))
    return reuse, both


@pytest.mark.parametrize("name", ["c1_fixture", "c2_fixture", "c3_fixture"])
def test_jacobian_bit_identical_with_half_the_work(engine, name):
    d = load_case(name)
    a, b = _pair(engine, d["cfg"])
    sa, sb = {}, {}
    Ja = a.jacobian(d["in0"], d["out0"], stats=sa)
    Jb = b.jacobian(d["in0"], d["out0"], stats=sb)
    assert np.array_equal(Ja, Jb)
    assert sa["shoots"] == sb["shoots"]
    assert sa["rhs_evals"] < 0.6 * sb["rhs_evals"], (sa["rhs_evals"], sb["rhs_evals"])
    a.close()
    b.close()


def test_column_ranges_across_block_edges(engine):
    d = load_case("c3_fixture")
    a, b = _pair(engine, d["cfg"])
    nn = a.nn
    for c0, c1 in [(0, 8), (nn // 3 - 4, nn // 3 + 4), (2 * nn // 3 - 1, 2 * nn // 3 + 5), (nn - 3, nn),
                   (nn - 2, nn + 1), (nn, nn + 1)]:
        out0 = d["out0"] if c0 < nn else None
        ca = a.jacobian_columns(d["in0"], out0, c0, c1)
        cb = b.jacobian_columns(d["in0"], out0, c0, c1)
        assert np.array_equal(ca, cb), (c0, c1)
    a.close()
    b.close()


def test_claim_order_does_not_change_bits(engine, monkeypatch):
    """The single-solve march hands its sweeps out from both ends of the
    longest-first list (by each slot's rank on its SM) unless
    PCC_MARCH_ENDS=0; which sweep runs where changes no result."""
    d = load_case("c3_fixture")
    a, b = _pair(engine, d["cfg"])
    st_ends, st_plain = {}, {}
    J_ends = a.jacobian(d["in0"], d["out0"], stats=st_ends)
    monkeypatch.setenv("PCC_MARCH_ENDS", "0")
    J_plain = a.jacobian(d["in0"], d["out0"], stats=st_plain)
    J_both = b.jacobian(d["in0"], d["out0"])
    assert np.array_equal(J_ends, J_plain) and np.array_equal(J_ends, J_both)
    assert st_ends["rhs_evals"] == st_plain["rhs_evals"]
    a.close()
    b.close()


def test_predictor_jacobian_bit_identical(engine):
    d = load_case("c2_fixture")
    a, b = _pair(engine, d["cfg"], IRKPredictor=True)
    assert np.array_equal(a.jacobian(d["in0"], d["out0"]), b.jacobian(d["in0"], d["out0"]))
    a.close()
    b.close()


def test_batch_and_newton_bit_identical(engine):
    c1, c2 = load_case("c1_newton"), load_case("c2_newton")
    a1, b1 = _pair(engine, c1["cfg"], PrecisionNewton=1e-12, MaxIterNewton=6)
    a2, b2 = _pair(engine, c2["cfg"], PrecisionNewton=float(c2["tol"]), MaxIterNewton=6)
    out1, out2 = a1.shoot(c1["in0"]), a2.shoot(c2["in0"])
    assert np.array_equal(out1, b1.shoot(c1["in0"]))
    Ja = engine.jacobian_batch([a1, a2], [c1["in0"], c2["in0"]], [out1, out2])
    Jb = engine.jacobian_batch([b1, b2], [c1["in0"], c2["in0"]], [out1, out2])
    assert all(np.array_equal(x, y) for x, y in zip(Ja, Jb))
    assert np.array_equal(Ja[0], a1.jacobian(c1["in0"], out1))
    xa, sta = engine.newton_solve([a1, a2], [c1["in0"], c2["in0"]], precision=1)
    xb, stb = engine.newton_solve([b1, b2], [c1["in0"], c2["in0"]], precision=1)
    for x, y, p, q in zip(xa, xb, sta, stb):
        assert np.array_equal(x, y)
        assert p["state"] == q["state"] == "CONVERGED"
        assert p["iterations"] == q["iterations"]
        assert p["err"] == q["err"]
    for s in (a1, b1, a2, b2):
        s.close()


def test_failure_reports_identical(engine):
    """With too few IRK iterations allowed the sweeps fail; both schedules name
    the same first failing column, side and grid index."""
    import pcc

    d = load_case("c1_fixture")
    for max_irk in (2, 4):
        a, b = _pair(engine, d["cfg"], MaxIterIRK=max_irk)
        reports = []
        for s in (a, b):
            st = {}
            with pytest.raises(pcc.PccError) as e:
                s.jacobian(d["in0"], d["out0"], stats=st)
            reports.append((e.value.status, st["fail_column"], st["fail_side"], st["fail_grid_index"]))
        assert reports[0] == reports[1], reports
        assert reports[0][1] >= 0
        a.close()
        b.close()
