"""The CPU oracle pinned to the reference.

* test/test_init_gen.cpp golden vectors (the reference's own known answers):
  pack/unpack round trip and both Taylor expansions at Ntau=128, D=4.
* Fixtures produced by the compiled reference (tests/golden/make_golden.py):
  unpack, expansions, RHS, single IRK steps, the base shoot and Jacobian
  columns at the configurations the GPU is benchmarked on.
* Known-answer tests replacing the two unusable reference tests
  (test_fft.cpp assumes the e^{-i} forward convention; test_lapack.cpp has an
  inconsistent right-hand side): a DFT of sin/exp under the reference's
  e^{+i}/N forward convention, and dgesv against numpy.
"""
import numpy as np
import pytest

from conftest import GOLDEN, load_case, rel_err


def test_init_gen_goldens(oracle):
    g = np.load(GOLDEN / "init_gen_128.npz")
    n, dim, delta = int(g["ntau"]), float(g["dim"]), float(g["delta"])
    z = oracle.pack(n, g["Up"], g["psic"], g["fc"])
    up, psic, fc = oracle.unpack(n, z)
    # relative tolerances: a different FFT than FFTW rounds differently (the
    # reference's 1e-15 absolute assert on psi_c ~ 168 is below round-off)
    assert rel_err(up, g["Up_unpack_ref"]) < 1e-13
    assert rel_err(psic, g["psic_unpack_ref"]) < 1e-13
    assert rel_err(fc, g["fc_unpack_ref"]) < 1e-13
    yl = oracle.left_expansion(n, dim, float(g["xl"]), fc, psic, delta)
    yr = oracle.right_expansion(n, dim, float(g["xr"]), up, delta)
    assert rel_err(yl, g["Yleft_ref"]) < 1e-13
    assert rel_err(yr, g["Yright_ref"]) < 1e-13


def test_dft_convention(oracle):
    """SpectralTransformer forward = e^{+i}, scaled 1/N (SpectralTransformer.cpp:33,57-72)."""
    import ctypes

    n = 16
    t = np.arange(n)
    x = np.sin(2 * np.pi * t / n)
    out = np.zeros(2 * n)
    oracle.lib.orc_forward_real(n, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    X = out[0::2] + 1j * out[1::2]
    expect = np.zeros(n, complex)
    expect[1], expect[n - 1] = 0.5j, -0.5j  # e^{+i}: sin -> +i/2 at k=1
    assert np.max(np.abs(X - expect)) < 1e-15
    assert np.allclose(X, np.conj(np.fft.fft(x)) / n, atol=1e-15)
    y = np.exp(2j * np.pi * 3 * t / n)
    buf = np.empty(2 * n)
    buf[0::2], buf[1::2] = y.real, y.imag
    oracle.lib.orc_dft(n, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), +1)
    Y = (buf[0::2] + 1j * buf[1::2]) / n
    assert abs(Y[n - 3] - 1) < 1e-14 and np.sum(np.abs(Y)) - 1 < 1e-13


def test_dgesv_known_answer(oracle):
    rng = np.random.default_rng(7)
    a = rng.standard_normal((40, 40)) + 40 * np.eye(40)
    xt = np.arange(1.0, 41.0)
    x, st = oracle.dgesv(a, a @ xt)
    assert st == 0
    assert np.max(np.abs(x - xt)) < 1e-12
    sing = np.ones((3, 3))
    _, st = oracle.dgesv(sing, np.ones(3))
    assert st != 0


@pytest.mark.parametrize("name", ["c1_fixture", "c1_perturbed", "c2_fixture", "c3_fixture"])
def test_boundary_and_rhs_vs_reference(oracle, name):
    d = load_case(name)
    cfg = d["cfg"]
    n, dim = cfg["Ntau"], cfg["Dim"]
    nn = 3 * n // 4
    z = d["in0"].copy()
    delta = z[2 * nn // 3 + 2]
    z[2 * nn // 3 + 2] = 0.0
    up, psic, fc = oracle.unpack(n, z)
    assert rel_err(up, d["unpack_up"]) < 1e-13
    assert rel_err(psic, d["unpack_psic"]) < 1e-13
    assert rel_err(fc, d["unpack_fc"]) < 1e-13
    assert rel_err(oracle.left_expansion(n, dim, cfg["XLeft"], fc, psic, delta), d["y_left"]) < 1e-12
    assert rel_err(oracle.right_expansion(n, dim, cfg["XRight"], up, delta), d["y_right"]) < 1e-12
    for y, x, dy in zip(d["rhs_y"], d["rhs_x"], d["rhs_dy"]):
        # the RHS divides by F - x, which is ~1e-3 near the horizon
        assert rel_err(oracle.rhs(n, dim, y, x), dy) < (1e-11 if x > 0.95 else 1e-13)
    for y, (xa, xb), yo, its in zip(d["irk_y"], d["irk_x"], d["irk_out"], d["irk_its"]):
        out, k, conv = oracle.irk_step(n, dim, cfg["SchemeIRK"], cfg["PrecisionIRK"], cfg["MaxIterIRK"], y, xa, xb)
        assert conv
        assert rel_err(out, yo) < 1e-13
        assert abs(k - int(its)) <= 1


def test_grid_vs_reference(oracle):
    for name in ["c1_fixture", "c3_fixture"]:
        d = load_case(name)
        assert rel_err(oracle.grid(d["cfg"]), d["grid"]) < 1e-15


def test_shoot_and_columns_vs_reference(oracle):
    """Base shoot and two Jacobian columns at C1 (Ntau=128, 1000+1000)."""
    d = load_case("c1_perturbed")
    out0, st, evals = oracle.shoot(d["cfg"], d["in0"])
    assert st == 0 and evals > 0
    # the shoot output is a ~1e-7 mismatch of O(1) states: FFT round-off of two
    # faithful FP64 implementations leaves ~1e-12 absolute differences
    assert np.max(np.abs(out0 - d["out0"])) < 1e-10
    cols, st, _ = oracle.jacobian_columns(d["cfg"], d["in0"], d["out0"], 0, 2)
    assert st == 0
    # eps = 1e-7 amplifies those differences to ~1e-6 of max|J|
    scale = np.max(np.abs(d["jac_cols"]))
    assert np.max(np.abs(cols - d["jac_cols"][:, :2])) / scale < 2e-5


def test_newton_update_reference_consistent(oracle):
    """The fixture's Newton update equals dgesv on the fixture's J (oracle LU)."""
    d = load_case("c1_perturbed")
    dx, st = oracle.dgesv(d["jac_cols"], -d["out0"])
    assert st == 0
    assert rel_err(dx, d["newton_dx"]) < 1e-9


def test_resample_oracle_matches_reference_script():
    """oracle_py.double_field against the reference's create_simulation_data.py
    double() (golden vectors made by importing the script)."""
    import oracle_py

    d = np.load(GOLDEN / "ref_resample_128.npz")
    for f in ["fc", "psic", "Up"]:
        x = d[f + "_128"]
        for n in [256, 512, 1024]:
            x = oracle_py.double_field(x)
            assert np.array_equal(x, d[f"{f}_{n}"]), (f, n)


def test_suite_goldens_and_quadratic_seeding():
    """The reference's continuation run (tests/golden/make_suite_golden.py):
    every dimension converged, and the quadratic seed of D_i (i >= 3) from the
    previous three converged ones (oracle_py restatement of main.cpp:300-354)
    lies close to the converged D_i the reference then found."""
    import oracle_py

    g = np.load(GOLDEN / "ref_suite_128.npz")
    for b in ["up", "down"]:
        assert g[f"{b}_converged"].all()
        dims = [float(k) for k in g[f"{b}_keys"]]
        assert (np.diff(dims) != 0).all()
        for i in range(3, len(dims)):
            prev = [dims[i - 1], dims[i - 2], dims[i - 3]]
            for f, tol in [("fc", 1e-5), ("Up", 1e-4), ("psic", 1e-3), ("delta", 1e-6)]:
                v = g[f"{b}_{f}"]
                seed = oracle_py.quadratic_extrapolate(prev, np.array([v[i - 1], v[i - 2], v[i - 3]]), dims[i])
                assert np.max(np.abs(seed - v[i])) / np.max(np.abs(v[i])) < tol, (b, i, f)
