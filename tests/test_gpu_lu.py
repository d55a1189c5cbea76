"""The dense Newton solve (NewtonSolver::solveLinearSystem, NewtonSolver.cpp:
739-757: LAPACKE_dgesv) at the benchmark's sizes: FP64, and FP32 + FP64
refinement with the FP32 trailing updates on the tensor cores (tcgen05,
TF32 high/low split) or, with PCC_LU_TC=0, on the CUDA cores.

Checks: the solution against LAPACK dgesv (numpy) on the reference's own
Jacobians (C1: n = 96, cond 3.3e6; C2: n = 384, cond 5.4e7) and on seeded
matrices of the C3 order (n = 768) and the largest order a solve has
(n = 1536, Ntau 2048), both with cond 1e6.  Two backward-stable solves of
the same system differ by up to about cond * eps, so the FP64 and the mixed
solution must each lie within 10 cond eps of dgesv's (relative, 2-norm); the
mixed solve must refine without falling back to FP64, in a few sweeps; both
FP32 update paths are held to the same bound."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_case

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _systems():
    d = load_case("c1_perturbed")
    yield "c1_reference_J", d["jac_cols"], -d["out0"]
    if (GOLDEN / "ref_c2_newton.npz").exists():
        d = load_case("c2_newton")
        yield "c2_reference_J", d["jacobian"], -d["out0"]
    rng = np.random.default_rng(768)
    for n in (768, 1536):
        # graded singular values 1 .. 1e-6: the conditioning of the Newton Jacobians
        u, _ = np.linalg.qr(rng.standard_normal((n, n)))
        v, _ = np.linalg.qr(rng.standard_normal((n, n)))
        A = (u * np.logspace(0, -6, n)) @ v.T
        yield f"seeded_{n}", A, rng.standard_normal(n)


@pytest.mark.parametrize("tc", ["1", "0"])
def test_lu_fp64_and_mixed_against_dgesv(engine, tc):
    old = os.environ.get("PCC_LU_TC")
    os.environ["PCC_LU_TC"] = tc
    try:
        for name, A, b in _systems():
            xn = np.linalg.solve(A, b)  # LAPACK dgesv
            tol = 10.0 * np.linalg.cond(A) * np.finfo(float).eps
            x64, r64 = engine.lu_solve(A, b, precision=0)
            assert _rel(x64, xn) < tol, (name, _rel(x64, xn), tol)
            xm, rm = engine.lu_solve(A, b, precision=1)
            assert rm["fell_back_to_fp64"] == 0, (name, rm)
            assert 1 <= rm["refinement_steps"] <= 8, (name, rm)
            assert _rel(xm, xn) < tol, (name, _rel(xm, xn), tol)
    finally:
        if old is None:
            os.environ.pop("PCC_LU_TC", None)
        else:
            os.environ["PCC_LU_TC"] = old


def test_lu_singular_is_reported(engine):
    """A zero column: dgesv's info > 0 becomes PCC_ERR_LU_SINGULAR."""
    import pcc

    A = np.random.default_rng(5).standard_normal((96, 96))
    A[:, 40] = 0.0
    for prec in (0, 1):
        with pytest.raises(pcc.PccError) as e:
            engine.lu_solve(A, np.ones(96), precision=prec)
        assert e.value.status == 7


def test_lu_order_above_limit_is_refused(engine):
    """The factorisation panel lives in shared memory, which bounds the order
    (3128); a larger system is refused before anything is allocated."""
    import pcc

    n = 3200
    with pytest.raises(pcc.PccError) as e:
        engine.lu_solve(np.eye(n), np.ones(n), precision=0)
    assert e.value.status == pcc.PCC_ERR_INVALID_ARG
