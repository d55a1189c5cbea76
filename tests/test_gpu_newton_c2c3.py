"""Parity at the benchmark's sizes: C2 (Ntau 512, 3000 + 3000 points) and C3
(Ntau 1024, 4000 + 4000 points, the benchmarked configuration).

* The benchmark's own C3 input (bench.workload: seed 1024, amplitude 0.1 around
  the packed near-solution): its base shoot and 24 Jacobian columns against
  the compiled reference on that same input (ref_c3_seed1024.npz).
* The reference's Newton loop (NewtonSolver.cpp:279-366) from a seeded
  relative perturbation of the near-solution (ref_c2_newton.npz,
  ref_c256_newton.npz at Ntau 256, ref_c3_newton.npz): the first Newton step and the converged solution,
  through the batched device-resident Newton loop (every shoot of an
  iteration in one persistent launch, the update on the device), with the
  FP64 and the mixed-precision solve.

Tolerances, as for C1 (tests/test_gpu_parity.py): Jacobian entries 2e-5 of
max |J| (EpsNewton = 1e-8 amplifies shoot round-off); one Newton step's Delta
1e-7 relative (it inherits that noise through the solve); the converged
Delta* 1e-10 relative (F(x*) = 0 fixes x* independently of the Jacobian's
noise); the converged free data 1e-6 relative (determined only to
||J^-1|| ||dF||); the LU update on the reference's own J within
max(1e-8, 10 cond(J) eps) of LAPACK dgesv's (two backward-stable solves of
one system differ by about cond eps).
"""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, REPO, load_case


def _have(name, done=True):
    p = GOLDEN / f"ref_{name}.npz"
    if not p.exists():
        return False
    return not done or int(np.load(p).get("done", 1)) == 1


def _islot(x):
    return 2 * x.size // 3 + 2


def test_bench_input_fixture_is_the_benchmarked_input():
    """The fixture holds exactly the free data bench.py times (CPU check)."""
    sys.path.insert(0, str(REPO))
    import bench

    d = load_case("c3_seed1024")
    cfg, in0 = bench.workload(int(d["seed"]), float(d["amp"]))
    assert np.array_equal(in0, d["in0"])
    assert {k: cfg[k] for k in ("Ntau", "NLeft", "NRight", "Dim", "EpsNewton")} == \
        {k: d["cfg"][k] for k in ("Ntau", "NLeft", "NRight", "Dim", "EpsNewton")}


@pytest.mark.gpu
def test_bench_input_shoot_and_jacobian_columns(engine):
    import pcc

    d = load_case("c3_seed1024")
    s = engine.solve(pcc.SolveDesc.from_config(d["cfg"]))
    out0 = s.shoot(d["in0"])
    assert np.max(np.abs(out0 - d["out0"])) < 1e-10
    Jr = d["jac_cols"]
    idx = [int(c) for c in d["jac_idx"]]
    J = np.concatenate([s.jacobian_columns(d["in0"], d["out0"], 0, 16),
                        s.jacobian_columns(d["in0"], d["out0"], 508, 516)], axis=1)
    assert idx == list(range(16)) + list(range(508, 516))
    assert np.max(np.abs(J - Jr)) / np.max(np.abs(Jr)) < 2e-5
    s.close()


def _newton_solve(engine, d, precision, tol):
    import pcc

    cfg = dict(d["cfg"], PrecisionNewton=tol, MaxIterNewton=12)
    s = engine.solve(pcc.SolveDesc.from_config(cfg))
    xs, states = engine.newton_solve([s], [d["in0"]], precision=precision)
    s.close()
    return xs[0], states[0]


def _newton_first_step(engine, d, precision):
    import pcc

    cfg = dict(d["cfg"], PrecisionNewton=1e-30, MaxIterNewton=100)
    s = engine.solve(pcc.SolveDesc.from_config(cfg))
    s.newton_begin(d["in0"])
    st = engine.newton_iterate([s], precision=precision)[0]
    x1, _ = s.newton_result()
    s.close()
    return x1, st


NEWTON = [c for c in ("c2_newton", "c256_newton") if _have(c)]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NEWTON)
@pytest.mark.parametrize("precision", [0, 1])
def test_newton_step_c2(engine, name, precision):
    d = load_case(name)
    x1, st = _newton_first_step(engine, d, precision)
    i = _islot(x1)
    assert abs(st["err"] / float(d["newton_err"]) - 1) < 1e-6
    assert abs(x1[i] / d["newton_in1"][i] - 1) < 1e-7
    assert np.linalg.norm(x1 - d["newton_in1"]) / np.linalg.norm(d["newton_in1"]) < 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("name", NEWTON)
@pytest.mark.parametrize("precision", [0, 1])
def test_lu_update_on_reference_jacobian_c2(engine, name, precision):
    """The dense solve alone on the reference's own J (384 x 384 at Ntau 512,
    192 x 192 at Ntau 256) against the reference's dgesv step, to 10 cond eps."""
    d = load_case(name)
    J = d["jacobian"]
    dx, rep = engine.lu_solve(J, -d["out0"], precision=precision)
    tol = max(1e-8, 10.0 * np.linalg.cond(J) * np.finfo(float).eps)
    assert np.linalg.norm(dx - d["newton_dx"]) / np.linalg.norm(d["newton_dx"]) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("name", NEWTON)
@pytest.mark.parametrize("precision", [0, 1])
def test_newton_converged_c2(engine, name, precision):
    d = load_case(name)
    x, st = _newton_solve(engine, d, precision, float(d["tol"]))
    assert st["state"] == "CONVERGED", st
    ref = d["x_star"]
    i = _islot(ref)
    assert abs(x[i] / ref[i] - 1) < 1e-10
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-6


@pytest.mark.gpu
@pytest.mark.skipif(not _have("c3_newton", done=False), reason="ref_c3_newton.npz not generated")
@pytest.mark.parametrize("precision", [0, 1])
def test_newton_step_c3(engine, precision):
    d = load_case("c3_newton")
    x1, st = _newton_first_step(engine, d, precision)
    i = _islot(x1)
    assert abs(st["err"] / float(d["newton_err"]) - 1) < 1e-6
    assert abs(x1[i] / d["newton_in1"][i] - 1) < 1e-7
    assert np.linalg.norm(x1 - d["newton_in1"]) / np.linalg.norm(d["newton_in1"]) < 1e-2


@pytest.mark.gpu
@pytest.mark.skipif(not _have("c3_newton"), reason="ref_c3_newton.npz not finished")
@pytest.mark.parametrize("precision", [0, 1])
def test_newton_converged_c3(engine, precision):
    """The north-star target: at Ntau 1024 with 8000 points the batched
    mixed-precision (and FP64) Newton loop reaches the reference's Delta* to
    1e-10 relative."""
    d = load_case("c3_newton")
    x, st = _newton_solve(engine, d, precision, float(d["tol"]))
    assert st["state"] == "CONVERGED", st
    ref = d["x_star"]
    i = _islot(ref)
    assert abs(x[i] / ref[i] - 1) < 1e-10
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-6
