"""Failure parity of the benchmark's C3 free data (bench.workload at
amplitude 0.1): the seeds bench.py skips because their base shoot does not
converge fail on the compiled reference too, on the same side, at the same
step (tests/golden/make_c3_seed_failures_golden.py: the reference's
ShootingSolver exits naming the failing step's starting grid index; the
engine reports it as fail_grid_index, within one step as the IRK
fixed-point iteration's last rounding may differ).  Seed 1031, which the
bench uses, converges on both."""
import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_c3_seed_failures_match_reference(engine):
    import pcc

    d = np.load(GOLDEN / "ref_c3_seed_failures.npz")
    cfg = json.loads(str(d["config"]))
    s = engine.solve(pcc.SolveDesc.from_config(cfg))
    for seed, in0, side, gi in zip(d["seeds"], d["in0"], d["side"], d["grid_index"]):
        st = {}
        if side < 0:
            s.shoot(in0, stats=st)
            assert st["fail_column"] == -1, seed
            continue
        with pytest.raises(pcc.PccError) as e:
            s.shoot(in0, stats=st)
        assert e.value.status == 4, seed  # PCC_ERR_IRK_NO_CONVERGENCE
        assert st["fail_side"] == side, (seed, st, side)
        assert abs(st["fail_grid_index"] - int(gi)) <= 1, (seed, st["fail_grid_index"], int(gi))
    s.close()
