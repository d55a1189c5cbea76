"""Dimension continuation (the reference's multiple-run mode, src/main.cpp:
245-378) through cc_b200 -m, against the reference's own cc_openmp -m run on
the same suites (tests/golden/make_suite_golden.py); and spectral resampling
(scripts/create_simulation_data.py:37-58) against the reference script.

Each dimension converges to PrecisionNewton = 1e-12 on both sides, so the
echoing period agrees to the parity tolerance (1e-10 relative) and the free
data to the Newton noise floor, whatever the seeds were."""
import json
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu


def test_resample_matches_reference_script(engine):
    d = np.load(GOLDEN / "ref_resample_128.npz")
    rows = np.array([d["fc_128"], d["psic_128"], d["Up_128"]])
    for n in [256, 512, 1024]:
        out = engine.resample(rows, n)
        for i, f in enumerate(["fc", "psic", "Up"]):
            ref = d[f"{f}_{n}"]
            assert np.max(np.abs(out[i] - ref)) / np.max(np.abs(ref)) < 1e-13, (f, n)


def _suite_file(path, g, branch):
    cfg = json.loads(str(g["config"]))
    seed = json.loads(str(g["seed_ic"]))
    out = {}
    for k, key in enumerate(g[f"{branch}_keys"]):
        c = dict(cfg)
        c["Dim"] = float(key)
        c["Converged"] = False
        c["Initial_Conditions"] = seed if k == 0 else {"Delta": None, "fc": None, "psic": None, "Up": None}
        out[str(key)] = c
    path.write_text(json.dumps(out))


def _check_against_reference(res, g, branch):
    for k, key in enumerate(g[f"{branch}_keys"]):
        r = res[str(key)]
        assert r["Converged"] is True, key
        ref_delta = g[f"{branch}_delta"][k]
        assert abs(r["Initial_Conditions"]["Delta"] / ref_delta - 1) < 1e-10, (key, r["Initial_Conditions"]["Delta"],
                                                                               ref_delta)
        for f in ["fc", "psic", "Up"]:
            ref = g[f"{branch}_{f}"][k]
            got = np.asarray(r["Initial_Conditions"][f])
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-6, (key, f)


def test_suite_continuation_matches_reference(tmp_path):
    g = np.load(GOLDEN / "ref_suite_128.npz")
    cli = str(PKG / "cc_b200")
    up, down = tmp_path / "up.json", tmp_path / "down.json"
    _suite_file(up, g, "up")
    _suite_file(down, g, "down")
    # both branches in lockstep, their Newton solves batched together
    r = subprocess.run([cli, "-m", "--suite", str(up), "asc", "--suite", str(down), "desc"], capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    res_up, res_down = json.loads(up.read_text()), json.loads(down.read_text())
    _check_against_reference(res_up, g, "up")
    _check_against_reference(res_down, g, "down")
    # the reference's own form, one suite: the same bits as in lockstep
    solo = tmp_path / "solo.json"
    _suite_file(solo, g, "up")
    r = subprocess.run([cli, "-m", "-r", "-i", str(solo)], capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    res_solo = json.loads(solo.read_text())
    for key in g["up_keys"]:
        assert res_solo[str(key)]["Initial_Conditions"] == res_up[str(key)]["Initial_Conditions"], key
