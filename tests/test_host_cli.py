"""The C++ host layer (NewtonSolver / SimulationConfig over the C ABI) through
its command line, which mirrors the reference's src/main.cpp single-run and
benchmark modes: the result dictionary is written back over the input JSON
with the reference's keys (NewtonSolver.cpp:775-816)."""
import json
import subprocess

import numpy as np
import pytest

from conftest import PKG, load_case

pytestmark = pytest.mark.gpu


def _config_file(tmp_path, engine, case="c1_newton"):
    d = load_case(case)
    cfg = dict(d["cfg"])
    n = cfg["Ntau"]
    nn = 3 * n // 4
    z = d["in0"].copy()
    delta = z[2 * nn // 3 + 2]
    z[2 * nn // 3 + 2] = 0.0
    up, psic, fc = engine.unpack(n, z)
    cfg["Initial_Conditions"] = {"Delta": delta, "fc": fc.tolist(), "psic": psic.tolist(), "Up": up.tolist()}
    cfg["MaxIterNewton"] = 12
    # PrecisionNewton = 1e-14 is below the round-off floor of this map (the
    # residual of the reference's own loop stalls near 3e-13), so the run uses
    # an attainable tolerance
    cfg["PrecisionNewton"] = 1e-12
    p = tmp_path / "sim.json"
    p.write_text(json.dumps(cfg))
    return p, d


def test_pack_unpack_round_trip(engine):
    d = load_case("c1_perturbed")
    n = 128
    z = d["in0"].copy()
    z[2 * 96 // 3 + 2] = 0.0
    up, psic, fc = engine.unpack(n, z)
    assert np.max(np.abs(up - d["unpack_up"])) < 1e-12
    z2 = engine.pack(n, up, psic, fc)
    keep = np.ones(96, bool)
    keep[[2 * 96 // 3 + 1, 2 * 96 // 3 + 2]] = False  # DC imaginary/Nyquist slot, Delta slot
    assert np.max(np.abs(z2[keep] - z[keep])) < 1e-13


def test_expansions_from_fields(engine):
    d = load_case("c1_fixture")
    cfg = d["cfg"]
    delta = d["in0"][2 * 96 // 3 + 2]
    yl, yr = engine.expansions(128, cfg["Dim"], delta, cfg["XLeft"], cfg["XRight"], d["unpack_fc"],
                               d["unpack_psic"], d["unpack_up"])
    assert np.max(np.abs(yl - d["y_left"])) / np.max(np.abs(d["y_left"])) < 1e-12
    assert np.max(np.abs(yr - d["y_right"])) / np.max(np.abs(d["y_right"])) < 1e-12


def test_dft_convention(engine):
    x = np.exp(2j * np.pi * 3 * np.arange(64) / 64)
    X = engine.dft(x, +1)[0] / 64
    assert abs(X[64 - 3] - 1) < 1e-14  # e^{+i} forward: e^{+2 pi i 3 j/N} -> bin N-3
    assert np.max(np.abs(engine.dft(X * 64, -1)[0] / 64 - x)) < 1e-14


def test_cli_single_run_converges(engine, tmp_path):
    cli = PKG / "cc_b200"
    if not cli.exists():
        pytest.fail("cc_b200 was not built")
    p, d = _config_file(tmp_path, engine)
    r = subprocess.run([str(cli), "-s", "-i", str(p)], capture_output=True, text=True, timeout=600)
    out = json.loads(p.read_text())
    assert out["Converged"] is True, r.stdout[-2000:] + r.stderr[-2000:]
    assert out["mismatchNorm"] < 1e-11
    ref_delta = d["x_star"][2 * 96 // 3 + 2]
    assert abs(out["Initial_Conditions"]["Delta"] / ref_delta - 1) < 1e-10
    for key in ["Ntau", "Dim", "XLeft", "XMid", "XRight", "EpsNewton", "PrecisionNewton", "SlowError",
                "MaxIterNewton", "NLeft", "NRight", "SchemeIRK", "PrecisionIRK", "MaxIterIRK", "IterNewton"]:
        assert key in out, key
    assert len(out["Initial_Conditions"]["fc"]) == 128


def test_cli_benchmark_mode(engine, tmp_path):
    cli = PKG / "cc_b200"
    p, _ = _config_file(tmp_path, engine, "c1_fixture")
    cfg = json.loads(p.read_text())
    cfg["MaxIterNewton"] = 2
    cfg["PrecisionNewton"] = 1e-30  # two timed Newton steps, then the (expected) non-convergence exit
    p.write_text(json.dumps(cfg))
    r = subprocess.run([str(cli), "-b", "--benchmark-repetitions", "1", "-i", str(p)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 1 and "did not converge" in r.stderr
