"""The one- and three-stage Gauss-Legendre schemes (SchemeIRK 1 and 3,
ODEStepper.cpp:163-292 with the tableaux of ODEStepper's constructor) through
whole shoots and Jacobian columns, against the compiled reference on the C1
setup (ref_c1_scheme1.npz, ref_c1_scheme3.npz: tests/golden/make_golden.py
--cases c1_schemes).  Tolerances as for the two-stage scheme: single IRK
steps 1e-13 relative (iteration count within one), the shoot's mismatch
1e-10 absolute, Jacobian columns 2e-5 of max |J|."""
import numpy as np
import pytest

from conftest import load_case, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme", [1, 3])
def test_scheme_irk_shoot_and_columns(engine, scheme):
    import pcc

    d = load_case(f"c1_scheme{scheme}")
    cfg = d["cfg"]
    assert cfg["SchemeIRK"] == scheme
    out, its = engine.irk_step(cfg["Ntau"], cfg["Dim"], scheme, cfg["PrecisionIRK"], cfg["MaxIterIRK"], d["irk_y"],
                               d["irk_x"][:, 0], d["irk_x"][:, 1])
    for k in range(2):
        assert rel_err(out[k], d["irk_out"][k]) < 1e-13
        assert abs(int(its[k]) - int(d["irk_its"][k])) <= 1
    s = engine.solve(pcc.SolveDesc.from_config(cfg))
    st = {}
    out0 = s.shoot(d["in0"], stats=st)
    assert st["fail_column"] == -1
    assert np.max(np.abs(out0 - d["out0"])) < 1e-10
    Jr = d["jac_cols"]
    for k, c in enumerate(d["jac_idx"]):
        col = s.jacobian_columns(d["in0"], d["out0"], int(c), int(c) + 1)[:, 0]
        assert np.max(np.abs(col - Jr[:, k])) / np.max(np.abs(Jr)) < 2e-5, (scheme, c)
    s.close()
