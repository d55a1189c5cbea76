"""The Debug output of a Newton iteration (the base shoot's field snapshots,
ShootingSolver.cpp:85-97 and 128-138, and the Jacobian CSV,
NewtonSolver.cpp:337-341) through cc_b200, against the files the reference's
own cc_openmp wrote for the same input (tests/golden/make_debug_golden.py):
same file names, same snapshot keys, fields to the shoot's round-off level,
the Jacobian to the finite-difference parity tolerance."""
import json
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, PKG, load_case

pytestmark = pytest.mark.gpu


def test_debug_export_matches_reference(tmp_path):
    g = np.load(GOLDEN / "ref_debug_128.npz")
    cfg = json.loads(str(g["config"]))
    p = tmp_path / "sim.json"
    p.write_text(json.dumps(cfg))
    r = subprocess.run([str(PKG / "cc_b200"), "-s", "-i", str(p)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 1 and "did not converge" in r.stderr  # one iteration, as the reference
    fields = json.loads((tmp_path / str(g["fields_file"])).read_text())
    assert sorted(fields.keys()) == sorted(str(k) for k in g["keys"])
    for i, key in enumerate(g["keys"]):
        for q in ["A", "U", "V", "f"]:
            got = np.asarray(fields[str(key)][q])
            ref = g[q][i]
            assert got.shape == ref.shape, (key, q)
            assert np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300) < 1e-9, (key, q)
    J = np.loadtxt(tmp_path / str(g["jacobian_file"]), delimiter=",")
    assert J.shape == g["J"].shape
    assert np.max(np.abs(J - g["J"])) / np.max(np.abs(g["J"])) < 2e-5


def test_shoot_debug_keeps_the_shoot(engine):
    import pcc

    d = load_case("c1_fixture")
    s = engine.solve(pcc.SolveDesc.from_config(d["cfg"]))
    out, idx, fields = s.shoot_debug(d["in0"], 100)
    assert np.array_equal(out, s.shoot(d["in0"]))  # the same kernel, the same bits
    nl = d["cfg"]["NLeft"]
    assert idx[0] == 0 and idx[len(idx) // 2 - 1] == nl - 1  # left sweep ascending to its last step
    assert idx[-1] == nl + 1 and np.all(np.isfinite(fields)) and np.all(fields[:, 0] > 0)
