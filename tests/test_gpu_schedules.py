"""The march kernel's transform schedules at Ntau = 1024: single transforms
(0), paired (1) and paired with the warp-exchange length-512 transforms (2),
each forced through PCC_MARCH_SCHEDULE in a fresh process.  Every schedule
reproduces the reference's RHS evaluations (1e-12 relative; 1e-10 at
x > 0.95, where the RHS divides by F - x), its C3 base shoot (1e-10
absolute) and its Delta column of J (2e-5 of max |J|)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1] + "/parallel-critical-collapse_b200")
sys.path.insert(0, sys.argv[1] + "/tests")
import pcc
from conftest import load_case
eng = pcc.Engine(0)
d = load_case("c3_fixture")
cfg = d["cfg"]
out = {}
dy = eng.rhs_eval(1024, cfg["Dim"], d["rhs_y"], list(d["rhs_x"]))
out["rhs"] = float(max(np.max(np.abs(dy[k] - d["rhs_dy"][k])) / np.max(np.abs(d["rhs_dy"][k]))
                       * (0.01 if d["rhs_x"][k] > 0.95 else 1.0) for k in range(len(dy))))
s = eng.solve(pcc.SolveDesc.from_config(cfg))
st = {}
o = s.shoot(d["in0"], stats=st)
out["shoot"] = float(np.max(np.abs(o - d["out0"])))
col = s.jacobian_columns(d["in0"], d["out0"], 514, 515)[:, 0]
k = list(d["jac_idx"]).index(514)
out["col"] = float(np.max(np.abs(col - d["jac_cols"][:, k])) / np.max(np.abs(d["jac_cols"])))
out["rhs_evals"] = st["rhs_evals"]
print("RESULT " + json.dumps(out))
"""


@pytest.mark.parametrize("sched", ["0", "1", "2"])
def test_schedule_parity_c3(sched):
    env = dict(os.environ, PCC_MARCH_SCHEDULE=sched)
    r = subprocess.run([sys.executable, "-c", CHILD, str(REPO)], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads([x for x in r.stdout.splitlines() if x.startswith("RESULT ")][-1][7:])
    assert res["rhs"] < 1e-12, res
    assert res["shoot"] < 1e-10, res
    assert res["col"] < 2e-5, res
