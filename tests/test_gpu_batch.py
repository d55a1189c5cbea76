"""Batches of solves in one persistent launch and the device-resident Newton
loop (NewtonSolver::run, NewtonSolver.cpp:279-372).

The batch kernel runs each sweep in one sweep slot with the same arithmetic
whatever else is in the launch, so a solve's results are bit-identical alone
and in a mix.  Against the single-solve kernel the comparison is numerical:
the two kernels are compiled separately and may contract different
multiply-adds, and the finite-difference Jacobian amplifies ulp differences
of the shoots by 1/EpsNewton.
"""
import numpy as np
import pytest

from conftest import load_case, rel_err

pytestmark = pytest.mark.gpu


def _solve(engine, cfg, **over):
    import pcc

    c = dict(cfg)
    c.update(over)
    return engine.solve(pcc.SolveDesc.from_config(c))


def _islot(x):
    return 2 * x.size // 3 + 2


def test_jacobian_batch_alone_mix_and_single(engine):
    c1, c2 = load_case("c1_fixture"), load_case("c2_fixture")
    s1 = _solve(engine, c1["cfg"])
    s1b = _solve(engine, c1["cfg"])
    s2 = _solve(engine, c2["cfg"])
    in1, in2 = c1["in0"], c2["in0"]
    out1, out2 = s1.shoot(in1), s2.shoot(in2)
    import pcc

    st = pcc.Stats()
    J_alone = engine.jacobian_batch([s1], [in1], [out1])[0]
    J_mix = engine.jacobian_batch([s2, s1b], [in2, in1], [out2, out1], stats=st)
    assert np.array_equal(J_alone, J_mix[1])  # same bits alone and in the mix
    assert st.shoots == 96 + 384 and st.rhs_evals > 0
    assert rel_err(J_alone, s1.jacobian(in1, out1)) < 1e-6
    assert rel_err(J_mix[0], s2.jacobian(in2, out2)) < 1e-6
    # and against the reference's own columns (the fixture holds a subset)
    cols = c1["jac_idx"]
    assert rel_err(J_alone[:, cols], c1["jac_cols"]) < 2e-5


def test_jacobian_batch_rejects_duplicates_and_unbatchable(engine):
    import pcc

    c1 = load_case("c1_fixture")
    s = _solve(engine, c1["cfg"])
    out = s.shoot(c1["in0"])
    with pytest.raises(pcc.PccError):
        engine.jacobian_batch([s, s], [c1["in0"]] * 2, [out] * 2)
    s3 = _solve(engine, c1["cfg"], SchemeIRK=3)
    with pytest.raises(pcc.PccError) as e:
        engine.jacobian_batch([s3], [c1["in0"]], [out])
    assert e.value.status == 9


@pytest.mark.parametrize("precision", [0, 1])
def test_device_newton_converges_to_reference(engine, precision):
    """Delta* against the reference's converged Delta* to 1e-10 (the target);
    the first mismatch against the reference's first mismatch."""
    d = load_case("c1_newton")
    s = _solve(engine, d["cfg"], PrecisionNewton=1e-12, MaxIterNewton=12)
    s.newton_begin(d["in0"])
    first = engine.newton_iterate([s], precision=precision)[0]
    assert abs(first["err"] / d["history"][0, 0] - 1) < 1e-8
    assert first["iterations"] == 1 and first["state"] == "RUNNING"
    while True:
        st = engine.newton_iterate([s], precision=precision)[0]
        if st["state"] != "RUNNING":
            break
    assert st["state"] == "CONVERGED", st
    assert st["iterations"] <= 7
    x, fin = s.newton_result()
    ref = d["x_star"]
    i = _islot(ref)
    assert abs(x[i] / ref[i] - 1) < 1e-10
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-6
    if precision == 1:
        assert st["lu_refinement_steps"] >= 1


def test_device_newton_step_matches_host_step(engine):
    """One device iteration against pcc_newton_step (host-side update).  The
    two Jacobians come from separately compiled kernels; with cond(J) ~ 3e6 at
    this point their ulp-level differences move the step by ~1e-6 relative,
    and Delta by far less (the noise floor of one Newton step)."""
    d = load_case("c1_perturbed")
    s = _solve(engine, d["cfg"], MaxIterNewton=1)
    s.newton_begin(d["in0"])
    st = engine.newton_iterate([s])[0]
    assert st["state"] == "MAX_ITER" and st["iterations"] == 1
    x_dev, _ = s.newton_result()
    x_host, err, _, _ = s.newton_step(d["in0"])
    assert abs(st["err"] / err - 1) < 1e-12
    step_dev, step_host = x_dev - d["in0"], x_host - d["in0"]
    assert np.linalg.norm(step_dev - step_host) / np.linalg.norm(step_host) < 1e-4
    i = _islot(x_dev)
    assert abs(x_dev[i] / x_host[i] - 1) < 1e-9


def test_device_newton_same_alone_and_in_mix(engine):
    c1, c2 = load_case("c1_newton"), load_case("c2_fixture")
    a = _solve(engine, c1["cfg"], PrecisionNewton=1e-12, MaxIterNewton=3)
    xa, sa = engine.newton_solve([a], [c1["in0"]])
    a2 = _solve(engine, c1["cfg"], PrecisionNewton=1e-12, MaxIterNewton=3)
    b = _solve(engine, c2["cfg"], PrecisionNewton=1e-30, MaxIterNewton=1)
    xm, sm = engine.newton_solve([b, a2], [c2["in0"], c1["in0"]])
    assert np.array_equal(xa[0], xm[1])
    assert sa[0]["iterations"] == sm[1]["iterations"] and sa[0]["err"] == sm[1]["err"]
    assert sm[0]["state"] == "MAX_ITER" and sm[0]["iterations"] == 1


def test_device_newton_reports_irk_failure(engine):
    d = load_case("c1_fixture")
    ok = _solve(engine, d["cfg"], PrecisionNewton=1e-30, MaxIterNewton=1)
    bad = _solve(engine, d["cfg"], MaxIterIRK=1)
    xs, st = engine.newton_solve([ok, bad], [d["in0"], d["in0"]])
    assert st[1]["state"] == "IRK_FAILED" and st[1]["fail_column"] >= 0 and st[1]["fail_grid_index"] >= 0
    assert np.array_equal(xs[1], d["in0"])  # no update applied
    assert st[0]["state"] == "MAX_ITER"


def test_jacobian_columns_device_blocks(engine):
    """pcc_jacobian_columns_device: column blocks of J on the device, column-
    major, as a column-sharded build over several GPUs uses them; the same
    bits as the corresponding columns of pcc_jacobian."""
    import torch

    d = load_case("c1_fixture")
    s = _solve(engine, d["cfg"])
    nn = s.nn
    out0 = s.shoot(d["in0"])
    J = s.jacobian(d["in0"], out0)
    din = torch.tensor(d["in0"], dtype=torch.float64, device="cuda")
    dout = torch.tensor(out0, dtype=torch.float64, device="cuda")
    for c0, c1 in [(0, 40), (40, nn)]:
        cols = torch.zeros((c1 - c0) * nn, dtype=torch.float64, device="cuda")
        s.jacobian_columns_device(din.data_ptr(), dout.data_ptr(), c0, c1, cols.data_ptr())
        s.sync()
        assert np.array_equal(cols.cpu().numpy().reshape(c1 - c0, nn).T, J[:, c0:c1])


def test_jacobian_device_graph_replays(engine):
    """pcc_jacobian_device captures its build into a CUDA graph on the first
    call for a set of pointers and replays it afterwards: every replay gives
    the bits of pcc_jacobian, with valid timings and counters; new pointers
    are captured anew."""
    import torch

    d = load_case("c1_fixture")
    s = _solve(engine, d["cfg"])
    nn = s.nn
    out0 = s.shoot(d["in0"])
    J = s.jacobian(d["in0"], out0)
    din = torch.tensor(d["in0"], dtype=torch.float64, device="cuda")
    dout = torch.tensor(out0, dtype=torch.float64, device="cuda")
    dJ = torch.empty((nn, nn), dtype=torch.float64, device="cuda")
    dJ2 = torch.empty((nn, nn), dtype=torch.float64, device="cuda")
    for k, target in enumerate([dJ, dJ, dJ, dJ2]):  # capture, two replays, capture anew
        target.fill_(float("nan"))
        torch.cuda.synchronize()
        s.jacobian_device(din.data_ptr(), dout.data_ptr(), target.data_ptr())
        st = s.sync()
        assert np.array_equal(target.cpu().numpy(), J), k
        assert st["ms_sweep"] > 0 and st["rhs_evals"] > 0 and st["shoots"] == nn


def test_march_autotuner_picks_the_faster_schedule(engine, tmp_path, monkeypatch):
    """The autotuner times paired and single transform schedules on its probe
    and keeps the paired one unless the single one is more than 3 % faster;
    the choice lands in the cache file."""
    cache = tmp_path / "autotune.txt"
    monkeypatch.setenv("PCC_AUTOTUNE_CACHE", str(cache))
    t = engine.march_tuning(2048, 1)  # a shape no other test builds
    assert t["ms_pair"] > 0 and t["ms_single"] > 0
    assert t["pair"] == (0 if t["ms_single"] < 0.97 * t["ms_pair"] else 1)
    line = cache.read_text().strip().splitlines()[-1]
    assert line.split("\t")[1].split()[:3] == ["2048", "1", str(t["pair"])]
    assert engine.march_tuning(2048, 1) == t  # remembered
