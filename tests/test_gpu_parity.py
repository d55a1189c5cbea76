"""Parity of the CUDA path with the reference (golden fixtures produced by the
compiled reference) and with the C oracle, through the C ABI.

Tolerances.  All arithmetic is FP64.  RHS, expansions and single IRK steps
agree to round-off (<= 1e-12 relative; 1e-10 where the RHS divides by
F - x ~ 1e-3 near x = 1).  A shoot returns the ~1e-7 mismatch of O(1) states
after thousands of steps; two faithful FP64 implementations differ there by
~1e-12 absolute (the C oracle against the compiled reference: 1.1e-12), so
shoots are compared to 1e-10 absolute.  The finite difference with EpsNewton
= 1e-7 turns that into noise of ~1e-5 of max|J| (oracle against reference:
2.0e-6), so Jacobians are compared at matrix scale to 2e-5.  With cond(J) ~
3e6 one Newton step inherits that noise (oracle against reference: Delta
6e-10 relative); the parity target "Delta to 1e-10" is checked where it is
well posed, on the converged Newton solution, which F(x*) = 0 fixes
independently of Jacobian noise.  The converged free data are determined to
||J^-1|| ||dF|| ~ 1.5e5 * 1e-11, i.e. ~5e-8 relative, and are compared to 1e-6.
"""
import numpy as np
import pytest

from conftest import load_case, rel_err

pytestmark = pytest.mark.gpu

CASES = ["c1_fixture", "c1_perturbed", "c2_fixture", "c3_fixture", "c2048"]


def _solve(engine, cfg, **over):
    import pcc

    c = dict(cfg)
    c.update(over)
    return engine.solve(pcc.SolveDesc.from_config(c))


@pytest.mark.parametrize("name", CASES)
def test_rhs_parity(engine, name):
    d = load_case(name)
    cfg = d["cfg"]
    dy = engine.rhs_eval(cfg["Ntau"], cfg["Dim"], d["rhs_y"], d["rhs_x"])
    for k, x in enumerate(d["rhs_x"]):
        assert rel_err(dy[k], d["rhs_dy"][k]) < (1e-10 if x > 0.95 else 1e-12), (name, x)


def _resample_state(base, ntau):
    """A state of ntau/2 modes from one of base.size/2 (zero padding or
    truncation of the spectrum), the Delta slot kept."""
    y = np.zeros(ntau)
    m = min(base.size, ntau)
    y[: m // 2] = base[: m // 2]          # modes 0 .. m/4-1
    y[ntau - m // 2:] = base[base.size - m // 2:]  # the negative-frequency end
    y[4] = base[4]  # Delta
    return y


@pytest.mark.parametrize("ntau", [128, 256, 512, 1024, 2048])
def test_rhs_random_states_vs_oracle(engine, oracle, ntau):
    """Seeded perturbed states at every supported Ntau, including 256 and 2048."""
    d = load_case("c1_fixture")
    cfg = d["cfg"]
    rng = np.random.default_rng(ntau)
    base = d["y_left"]
    y = _resample_state(base, ntau) * (1 + 1e-3 * rng.standard_normal(ntau))
    y[4] = base[4]  # Delta
    xs = np.array([0.002, 0.05, 0.3])
    dy = engine.rhs_eval(ntau, cfg["Dim"], np.stack([y] * 3), xs)
    for k, x in enumerate(xs):
        assert rel_err(dy[k], oracle.rhs(ntau, cfg["Dim"], y, x)) < 1e-12, (ntau, x)


@pytest.mark.parametrize("name", CASES)
def test_irk_step_parity(engine, name):
    d = load_case(name)
    cfg = d["cfg"]
    out, its = engine.irk_step(cfg["Ntau"], cfg["Dim"], cfg["SchemeIRK"], cfg["PrecisionIRK"], cfg["MaxIterIRK"],
                               d["irk_y"], d["irk_x"][:, 0], d["irk_x"][:, 1])
    for k in range(2):
        assert rel_err(out[k], d["irk_out"][k]) < 1e-13
        assert abs(int(its[k]) - int(d["irk_its"][k])) <= 1


@pytest.mark.parametrize("scheme", [1, 3])
def test_irk_schemes_vs_oracle(engine, oracle, scheme):
    d = load_case("c1_fixture")
    cfg = d["cfg"]
    y, xa, xb = d["irk_y"][0], d["irk_x"][0, 0], d["irk_x"][0, 1]
    out, its = engine.irk_step(128, cfg["Dim"], scheme, 1e-15, 100, y[None], [xa], [xb])
    ref, k, conv = oracle.irk_step(128, cfg["Dim"], scheme, 1e-15, 100, y, xa, xb)
    assert conv
    assert rel_err(out[0], ref) < 1e-13
    assert abs(int(its[0]) - k) <= 1


@pytest.mark.parametrize("ntau,scheme", [(256, 2), (2048, 2), (2048, 1), (2048, 3), (1024, 1), (1024, 3)])
def test_irk_step_shapes_vs_oracle(engine, oracle, ntau, scheme):
    """One IRK step at the kernel shapes the fixtures do not reach: Ntau 256
    and 2048 (single transforms, 4 to 12 warps per sweep) and the one- and
    three-stage schemes at Ntau 1024 (paired transforms, up to 6 warps and
    one CTA per SM), from the C1 step state zero-padded to ntau modes."""
    d = load_case("c1_fixture")
    cfg = d["cfg"]
    y = _resample_state(d["irk_y"][0], ntau)
    xa, xb = d["irk_x"][0, 0], d["irk_x"][0, 1]
    out, its = engine.irk_step(ntau, cfg["Dim"], scheme, 1e-15, 100, y[None], [xa], [xb])
    ref, k, conv = oracle.irk_step(ntau, cfg["Dim"], scheme, 1e-15, 100, y, xa, xb)
    assert conv
    assert rel_err(out[0], ref) < 1e-12, (ntau, scheme)
    assert abs(int(its[0]) - k) <= 1, (ntau, scheme, int(its[0]), k)


@pytest.mark.parametrize("name", CASES)
def test_boundary_data_parity(engine, name):
    d = load_case(name)
    s = _solve(engine, d["cfg"])
    yl, yr = s.boundary_data(d["in0"])
    assert rel_err(yl, d["y_left"]) < 1e-12
    assert rel_err(yr, d["y_right"]) < 1e-12


def _interp_field(f, n):
    """Spectral (zero-padding) interpolation of a periodic real field to n samples."""
    c = np.fft.rfft(f)
    c2 = np.zeros(n // 2 + 1, dtype=complex)
    c2[: c.size - 1] = c[:-1]  # the old Nyquist term is dropped (a single cosine, ambiguous when padded)
    return np.fft.irfft(c2, n) * (n / f.size)


@pytest.mark.parametrize("ntau", [256, 1024, 2048])
def test_boundary_kernels_shapes_vs_oracle(engine, oracle, ntau):
    """Pack, unpack and both Taylor expansions at more samples than the C1
    fixture has: the C1 fields interpolated spectrally to ntau points."""
    d = load_case("c1_fixture")
    cfg = d["cfg"]
    up, psic, fc = (_interp_field(d[k], ntau) for k in ("unpack_up", "unpack_psic", "unpack_fc"))
    z = engine.pack(ntau, up, psic, fc)
    assert rel_err(z, oracle.pack(ntau, up, psic, fc)) < 1e-12
    up2, psic2, fc2 = engine.unpack(ntau, z)
    uo, po, fo = oracle.unpack(ntau, z)
    for a, b in ((up2, uo), (psic2, po), (fc2, fo)):
        assert rel_err(a, b) < 1e-12
    delta = float(d["in0"][2 * d["in0"].size // 3 + 2])
    yl, yr = engine.expansions(ntau, cfg["Dim"], delta, cfg["XLeft"], cfg["XRight"], fc, psic, up)
    assert rel_err(yl, oracle.left_expansion(ntau, cfg["Dim"], cfg["XLeft"], fc, psic, delta)) < 1e-12
    assert rel_err(yr, oracle.right_expansion(ntau, cfg["Dim"], cfg["XRight"], up, delta)) < 1e-12


def test_grid_parity(engine):
    d = load_case("c3_fixture")
    s = _solve(engine, d["cfg"])
    assert rel_err(s.grid(), d["grid"]) < 1e-15


@pytest.mark.parametrize("name", CASES)
def test_shoot_parity(engine, name):
    d = load_case(name)
    s = _solve(engine, d["cfg"])
    st = {}
    out0 = s.shoot(d["in0"], stats=st)
    assert st["rhs_evals"] > 0 and st["fail_column"] == -1
    # absolute: the outputs are the mismatch itself (~1e-7)
    assert np.max(np.abs(out0 - d["out0"])) < 1e-10, name
    assert abs(np.sqrt(np.mean(out0 ** 2)) / np.sqrt(np.mean(d["out0"] ** 2)) - 1) < 1e-3


def test_sweep_vs_oracle(engine, oracle):
    """integrateToMatchPoint of the reference's boundary states, both sides."""
    d = load_case("c1_fixture")
    cfg = d["cfg"]
    s = _solve(engine, cfg)
    st = {}
    y = s.sweep(np.stack([d["y_left"], d["y_right"]]), [0, 1], stats=st)
    yl_o, s0, _, e0 = oracle.sweep(cfg, d["y_left"], True)
    yr_o, s1, _, e1 = oracle.sweep(cfg, d["y_right"], False)
    assert s0 == 0 and s1 == 0
    assert np.max(np.abs(y[0] - yl_o)) < 1e-10
    assert np.max(np.abs(y[1] - yr_o)) < 1e-10
    # RHS evaluations counted on the device match the oracle's count closely
    assert abs(st["rhs_evals"] - (e0 + e1)) <= 0.01 * (e0 + e1)


def test_sweep_shapes_vs_oracle(engine, oracle):
    """Left sweeps of the C1 grid from the C1 boundary state zero-padded to
    more modes.  At Ntau 256 the march converges and matches the oracle; at
    Ntau 2048 the grid is too coarse for the stiffer spectrum, and both report
    the IRK failure at the same grid index (the reference exits there)."""
    import pcc

    d = load_case("c1_fixture")
    cfg = dict(d["cfg"], Ntau=256)
    y = _resample_state(d["y_left"], 256)
    yo, st_o, _, _ = oracle.sweep(cfg, y, True)
    assert st_o == 0
    out = _solve(engine, cfg).sweep(y[None], [0])
    assert np.max(np.abs(out[0] - yo)) < 1e-10

    cfg = dict(d["cfg"], Ntau=2048)
    y = _resample_state(d["y_left"], 2048)
    _, st_o, fail_o, _ = oracle.sweep(cfg, y, True)
    assert st_o != 0
    st = {}
    with pytest.raises(pcc.PccError) as e:
        _solve(engine, cfg).sweep(y[None], [0], stats=st)
    assert e.value.status == 4
    assert abs(st["fail_grid_index"] - fail_o) <= 1, (st["fail_grid_index"], fail_o)


@pytest.mark.parametrize("name", ["c1_fixture", "c1_perturbed"])
def test_jacobian_c1(engine, name):
    d = load_case(name)
    s = _solve(engine, d["cfg"])
    st = {}
    J = s.jacobian(d["in0"], d["out0"], stats=st)
    Jr = d["jac_cols"]
    assert np.max(np.abs(J - Jr)) / np.max(np.abs(Jr)) < 2e-5
    big = np.max(np.abs(Jr), axis=0) > 1e-2 * np.max(np.abs(Jr))  # columns above the noise level
    errs = [rel_err(J[:, k], Jr[:, k]) for k in np.nonzero(big)[0]]
    assert np.median(errs) < 1e-4
    assert st["shoots"] == 96


@pytest.mark.parametrize("name", ["c2_fixture", "c3_fixture"])
def test_jacobian_columns_c2_c3(engine, name):
    """Leading column of each field and the Delta column at Ntau = 512 and 1024."""
    d = load_case(name)
    s = _solve(engine, d["cfg"])
    Jr = d["jac_cols"]
    scale = np.max(np.abs(Jr))
    for k, c in enumerate(d["jac_idx"]):
        col = s.jacobian_columns(d["in0"], d["out0"], int(c), int(c) + 1)[:, 0]
        assert np.max(np.abs(col - Jr[:, k])) / scale < 2e-5, c


def test_jacobian_columns_c2048(engine):
    """Columns 0..7 at Ntau 2048 (8000 + 8000 points) in one launch."""
    d = load_case("c2048")
    s = _solve(engine, d["cfg"])
    Jr = d["jac_cols"]
    J = s.jacobian_columns(d["in0"], d["out0"], 0, Jr.shape[1])
    assert np.max(np.abs(J - Jr)) / np.max(np.abs(Jr)) < 2e-5


@pytest.mark.parametrize("precision", [0, 1])
def test_newton_step_c1(engine, precision):
    """One Newton iteration (NewtonSolver.cpp:298-358) against the reference's."""
    d = load_case("c1_perturbed")
    s = _solve(engine, d["cfg"])
    in1, err, st, rep = s.newton_step(d["in0"], precision=precision)
    nn = d["in0"].size
    islot = 2 * nn // 3 + 2
    assert abs(err / float(d["newton_err"]) - 1) < 1e-6
    # inherits the Jacobian's finite-difference noise (see the module docstring)
    assert abs(in1[islot] / d["newton_in1"][islot] - 1) < 1e-7
    assert np.linalg.norm(in1 - d["newton_in1"]) / np.linalg.norm(d["newton_in1"]) < 1e-2
    out1 = s.shoot(in1)
    r1, rr = np.sqrt(np.mean(out1 ** 2)), np.sqrt(np.mean(d["newton_out1"] ** 2))
    assert r1 < 2.0 * rr


@pytest.mark.parametrize("precision", [0, 1])
def test_newton_update_on_reference_jacobian(engine, precision):
    """The dense solve and damped update alone, on the reference's J and F:
    LAPACKE_dgesv semantics to round-off (FP64 LU, and FP32 LU + refinement)."""
    d = load_case("c1_perturbed")
    dx, rep = engine.lu_solve(d["jac_cols"], -d["out0"], precision=precision)
    assert np.linalg.norm(dx - d["newton_dx"]) / np.linalg.norm(d["newton_dx"]) < 1e-8
    err = np.sqrt(np.mean(d["out0"] ** 2))
    in1 = d["in0"] + min(1.0, d["cfg"]["SlowError"] / err) * dx
    nn = d["in0"].size
    assert abs(in1[2 * nn // 3 + 2] / d["newton_in1"][2 * nn // 3 + 2] - 1) < 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_newton_converged_solution_c1(engine, precision):
    """Newton iterations to the round-off floor; Delta* against the reference's
    converged Delta* to 1e-10 relative (the parity target), FP64 and mixed."""
    d = load_case("c1_newton")
    s = _solve(engine, d["cfg"])
    x = d["in0"].copy()
    nn = x.size
    islot = 2 * nn // 3 + 2
    errs = []
    for _ in range(8):
        x_next, err, st, rep = s.newton_step(x, precision=precision)
        errs.append(err)
        if err < 1e-12:
            break
        x = x_next
    assert min(errs) < 1e-12, errs
    ref_star = d["x_star"]
    assert abs(x[islot] / ref_star[islot] - 1) < 1e-10
    assert np.linalg.norm(x - ref_star) / np.linalg.norm(ref_star) < 1e-6


def test_lu_fp64_and_mixed(engine):
    d = load_case("c1_perturbed")
    J, b = d["jac_cols"], -d["out0"]
    x64, rep64 = engine.lu_solve(J, b, precision=0)
    xn = np.linalg.solve(J, b)
    assert np.linalg.norm(x64 - xn) / np.linalg.norm(xn) < 1e-9
    xm, repm = engine.lu_solve(J, b, precision=1)
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-9
    assert repm["refinement_steps"] >= 1


def test_irk_no_convergence_is_reported(engine):
    """MaxIterIRK = 1 cannot converge: the reference exits, we return a status."""
    import pcc

    d = load_case("c1_fixture")
    s = _solve(engine, d["cfg"], MaxIterIRK=1)
    with pytest.raises(pcc.PccError) as e:
        s.shoot(d["in0"])
    assert e.value.status == 4
    # the context stays usable
    s2 = _solve(engine, d["cfg"])
    out0 = s2.shoot(d["in0"])
    assert np.max(np.abs(out0 - d["out0"])) < 1e-10


def test_non_finite_free_data_is_refused(engine):
    """A NaN or an infinity in the free data handed in through host pointers
    is refused with PCC_ERR_NAN before any launch (the reference would run
    into an IRK failure and exit); the context stays usable."""
    import pcc

    d = load_case("c1_fixture")
    s = _solve(engine, d["cfg"])
    bad = d["in0"].copy()
    bad[7] = np.nan
    for call in (lambda: s.shoot(bad), lambda: s.jacobian(bad, d["out0"]),
                 lambda: s.jacobian(d["in0"], np.where(np.arange(bad.size) == 3, np.inf, d["out0"])),
                 lambda: engine.newton_solve([s], [bad])):
        with pytest.raises(pcc.PccError) as e:
            call()
        assert e.value.status == pcc.PCC_ERR_NAN
    out0 = s.shoot(d["in0"])
    assert np.max(np.abs(out0 - d["out0"])) < 1e-10


def test_invalid_arguments(engine):
    import pcc

    d = load_case("c1_fixture")
    for bad in [dict(Ntau=100), dict(NLeft=0), dict(XMid=0.9999), dict(SchemeIRK=4)]:
        with pytest.raises(pcc.PccError) as e:
            _solve(engine, d["cfg"], **bad)
        assert e.value.status == 1
