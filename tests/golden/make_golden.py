"""Generates the golden fixtures under tests/golden/ from the reference.

TEST INFRASTRUCTURE ONLY.  Run where the reference tree exists:

    python tests/golden/make_golden.py --reference <reference checkout> [--cases c1 c2 ...]

(--reference defaults to $PCC_REFERENCE_ROOT.)

Sources of truth:
  * test/test_init_gen.cpp (the reference's own golden vectors, parsed as text)
    -> init_gen_128.npz
  * the compiled reference (oracle/_ref/libpcc_ref.so, built by
    oracle/build_ref.sh from the reference's sources) run on the reference's
    data/simulation_4D_{128,512,1024}.json near-solutions and on seeded
    perturbations of them -> ref_<case>.npz

Each ref_<case>.npz holds the reference SimulationConfig (JSON string, with
the grid sizes the case uses), the packed Newton input in0 (Delta in slot
2*Nnewton/3+2), and the reference's outputs: boundary states, RHS
evaluations, single IRK steps, the base shoot, Jacobian columns and, where
the full Jacobian is present, the LAPACK Newton update.

Further cases:
  * c3_seed1024 -- the benchmark's own C3 input (bench.workload(1024, 0.1)):
    its base shoot and 24 reference Jacobian columns (0..15, 508..515);
  * c1_scheme1, c1_scheme3 -- C1 with SchemeIRK 1 and 3: shoot and four
    Jacobian columns;
  * c256_newton -- the Newton loop at Ntau 256 (2000 + 2000 points), as
    c2_newton;
  * c2048 -- Ntau 2048 with the data file's 8000 + 8000 points: boundary
    data, RHS, IRK steps, the base shoot and Jacobian columns 0..7;
  * c2_newton, c3_newton -- the reference's Newton loop
    (NewtonSolver.cpp:279-366) from a seeded 1e-3 / 1e-4 relative
    perturbation of the near-solution until the mismatch RMS is below 1e-12:
    the first step's Jacobian (C2 only; 4.7 MB at C3 is not committed), LAPACK
    update and next iterate, the residual/Delta history and the converged
    unknowns.  The C3 run takes hours on 8 cores; the file is rewritten after
    every iteration (key `done` = 0 until the loop has ended).
"""
import argparse
import json
import os
import re
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from ref_lib import RefLib  # noqa: E402

SEED = 20261203


def parse_init_gen(src):
    def arr(name, cplx=False):
        m = re.search(r"vec_(?:real|complex)\s+" + name + r"\s*=\s*\{(.*?)\};", src, re.S)
        body = re.sub(r"/\*.*?\*/", "", m.group(1))
        if cplx:
            pairs = re.findall(r"\{\s*([^,{}]+)\s*,\s*([^,{}]+)\s*\}", body)
            return np.array([[float(a), float(b)] for a, b in pairs]).reshape(-1)
        return np.array([float(x) for x in body.replace("\n", " ").split(",") if x.strip()])

    return {k: arr(k) for k in ["fc", "psic", "Up", "Up_unpack_ref", "psic_unpack_ref", "fc_unpack_ref"]} | {
        "Yleft_ref": arr("Yleft_ref", True), "Yright_ref": arr("Yright_ref", True)}


def config(ref_root, ntau, nl, nr):
    cfg = json.loads((ref_root / "data" / f"simulation_4D_{ntau}.json").read_text())
    cfg["NLeft"], cfg["NRight"] = nl, nr
    cfg["Verbose"] = False
    cfg["Debug"] = False
    return cfg


def packed_input(R, cfg):
    ic = cfg["Initial_Conditions"]
    n = cfg["Ntau"]
    z = R.pack(n, cfg["Dim"], ic["Delta"], ic["Up"], ic["psic"], ic["fc"])
    z[2 * len(z) // 3 + 2] = ic["Delta"]
    return z


def perturb(z, rel, rng):
    """Relative N(0, rel) perturbation of every free coefficient except Delta."""
    z = z.copy()
    islot = 2 * len(z) // 3 + 2
    noise = 1.0 + rel * rng.standard_normal(z.size)
    noise[islot] = 1.0
    return z * noise


def case(R, cfg, in0, name, jac_idx, threads, full_newton=False):
    n, D = cfg["Ntau"], cfg["Dim"]
    nn = 3 * n // 4
    out = {"config": json.dumps({k: v for k, v in cfg.items() if k != "Initial_Conditions"}), "in0": in0}
    z = in0.copy()
    delta = z[2 * nn // 3 + 2]
    z[2 * nn // 3 + 2] = 0.0
    up, psic, fc = R.unpack(n, D, delta, z)
    yl = R.left_expansion(n, D, cfg["XLeft"], fc, psic, delta)
    yr = R.right_expansion(n, D, cfg["XRight"], up, delta)
    out.update(unpack_up=up, unpack_psic=psic, unpack_fc=fc, y_left=yl, y_right=yr)
    xs = np.array([cfg["XLeft"], 0.01, 0.05, cfg["XMid"], 0.5, 0.9, cfg["XRight"]])
    states = np.stack([yl, yl, yl, yl, yr, yr, yr])
    out["rhs_x"] = xs
    out["rhs_y"] = states
    out["rhs_dy"] = np.stack([R.rhs(n, D, y, x) for y, x in zip(states, xs)])
    grid = R.grid(cfg)
    out["grid"] = grid
    steps = [(yl, grid[0], grid[1]), (yr, grid[-1], grid[-2])]
    irk = [R.irk_step(n, D, cfg["SchemeIRK"], cfg["PrecisionIRK"], cfg["MaxIterIRK"], y, a, b) for y, a, b in steps]
    out["irk_y"] = np.stack([s[0] for s in steps])
    out["irk_x"] = np.array([[s[1], s[2]] for s in steps])
    out["irk_out"] = np.stack([r[0] for r in irk])
    out["irk_its"] = np.array([r[1] for r in irk])
    t = time.time()
    out0 = R.shoot(cfg, in0)
    out["out0"] = out0
    out["t_shoot_s"] = time.time() - t
    if jac_idx is not None:
        jac_idx = list(jac_idx)
        t = time.time()
        out["jac_idx"] = np.array(jac_idx)
        out["jac_cols"] = np.concatenate([R.jacobian_columns(cfg, in0, out0, c, c + 1, 1) for c in jac_idx], axis=1) \
            if len(jac_idx) < 16 else R.jacobian_columns(cfg, in0, out0, jac_idx[0], jac_idx[-1] + 1, threads)
        out["t_jac_s"] = time.time() - t
        if full_newton and jac_idx == list(range(nn)):
            J = out["jac_cols"]
            dx = R.solve(J, -out0)
            err = np.sqrt(np.mean(out0 ** 2))
            fac = min(1.0, cfg["SlowError"] / err)
            in1 = in0 + fac * dx
            out.update(newton_dx=dx, newton_in1=in1, newton_err=err,
                       newton_out1=R.shoot(cfg, in1))
    np.savez_compressed(HERE / f"ref_{name}.npz", **out)
    print(name, {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items() if k != "config"})


def newton_to_convergence(R, cfg, in0, name, threads, iters=8):
    """The reference's Newton loop (NewtonSolver.cpp:279-366) run from in0:
    the converged solution and the residual history."""
    nn = in0.size
    x = in0.copy()
    hist = []
    for _ in range(iters):
        out = R.shoot(cfg, x)
        err = float(np.sqrt(np.mean(out ** 2)))
        hist.append([err, x[2 * nn // 3 + 2]])
        J = R.jacobian_columns(cfg, x, out, 0, nn, threads)
        dx = R.solve(J, -out)
        x = x + min(1.0, cfg["SlowError"] / err) * dx
    out = R.shoot(cfg, x)
    hist.append([float(np.sqrt(np.mean(out ** 2))), x[2 * nn // 3 + 2]])
    np.savez_compressed(HERE / f"ref_{name}.npz", config=json.dumps({k: v for k, v in cfg.items()
                                                                        if k != "Initial_Conditions"}),
                        in0=in0, x_star=x, history=np.array(hist))
    print(name, "history", hist)


def bench_input_case(R, threads):
    """The benchmark's C3 input (bench.workload: seed 1024, amplitude 0.1 around
    the packed near-solution) through the reference: base shoot and Jacobian
    columns 0..15 (the CPU-baseline sample) and 508..515 (the last f_c modes
    before and after Delta's slot 514)."""
    sys.path.insert(0, str(HERE.parents[1]))
    import bench  # the repository's benchmark: its workload() makes the input

    cfg, in0 = bench.workload(1024, 0.1)
    t = time.time()
    out0 = R.shoot(cfg, in0)
    idx = list(range(16)) + list(range(508, 516))
    cols = np.concatenate([R.jacobian_columns(cfg, in0, out0, 0, 16, threads),
                           R.jacobian_columns(cfg, in0, out0, 508, 516, threads)], axis=1)
    np.savez_compressed(HERE / "ref_c3_seed1024.npz", config=json.dumps(cfg), seed=1024, amp=0.1, in0=in0,
                        out0=out0, jac_idx=np.array(idx), jac_cols=cols, t_s=time.time() - t)
    print("c3_seed1024", cols.shape, f"{time.time() - t:.0f} s")


def newton_case(R, cfg, x0, name, threads, store_jacobian, tol=1e-12, max_iters=8):
    """The reference's Newton loop (NewtonSolver.cpp:279-366, which stops when
    the mismatch RMS drops below PrecisionNewton; here `tol`) from x0, with a
    checkpoint after every iteration."""
    nn = x0.size
    islot = 2 * nn // 3 + 2
    base = {"config": json.dumps({k: v for k, v in cfg.items() if k != "Initial_Conditions"}), "in0": x0,
            "tol": tol}
    x = x0.copy()
    hist, extra = [], {}
    t0 = time.time()
    for it in range(max_iters):
        out = R.shoot(cfg, x)
        err = float(np.sqrt(np.mean(out ** 2)))
        hist.append([err, x[islot]])
        if it == 0:
            extra["out0"] = out
        elif it == 1:
            extra["newton_out1"] = out
        if err < tol:
            break
        J = R.jacobian_columns(cfg, x, out, 0, nn, threads)
        dx = R.solve(J, -out)
        fac = min(1.0, cfg["SlowError"] / err)
        if it == 0:
            extra.update(newton_dx=dx, newton_in1=x + fac * dx, newton_err=err)
            if store_jacobian:
                extra["jacobian"] = J
        x = x + fac * dx
        np.savez_compressed(HERE / f"ref_{name}.npz", **base, **extra, x_last=x, history=np.array(hist), done=0,
                            t_s=time.time() - t0)
        print(name, "iteration", it, "err", err, "Delta", hist[-1][1], f"{time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(HERE / f"ref_{name}.npz", **base, **extra, x_star=x, history=np.array(hist), done=1,
                        t_s=time.time() - t0)
    print(name, "history", hist, flush=True)


CASES = ["init_gen", "c1", "c2", "c3", "c3_seed1024", "c2_newton", "c3_newton", "c1_schemes", "c256_newton",
         "c2048"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PCC_REFERENCE_ROOT"),
                    help="reference checkout (default $PCC_REFERENCE_ROOT)")
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("--cases", nargs="+", choices=CASES, default=CASES[:5])
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set PCC_REFERENCE_ROOT")
    ref = Path(a.reference)
    if "init_gen" in a.cases:
        src = (ref / "test" / "test_init_gen.cpp").read_text()
        g = parse_init_gen(src)
        np.savez_compressed(HERE / "init_gen_128.npz", ntau=128, dim=4.0, delta=3.445501184653556, xl=0.001,
                            xr=0.999, **g)
    R = RefLib()
    rng = np.random.default_rng(SEED)
    if "c1" in a.cases:
        # C1: Ntau=128, 1000+1000 points, full Jacobian and Newton step, fixture and seeded perturbation
        cfg = config(ref, 128, 1000, 1000)
        z = packed_input(R, cfg)
        case(R, cfg, z, "c1_fixture", range(96), a.threads, full_newton=True)
        zp = perturb(z, 1e-3, rng)
        case(R, cfg, zp, "c1_perturbed", range(96), a.threads, full_newton=True)
        newton_to_convergence(R, cfg, zp, "c1_newton", a.threads)
    if "c2" in a.cases:
        # C2: Ntau=512, 3000+3000: base shoot and the leading column of each field plus Delta
        cfg = config(ref, 512, 3000, 3000)
        case(R, cfg, packed_input(R, cfg), "c2_fixture", [0, 128, 256, 258], a.threads)
    if "c3" in a.cases:
        # C3: Ntau=1024, 4000+4000: the same columns (Up mode 1, psi_c mode 1, f_c DC, Delta)
        cfg = config(ref, 1024, 4000, 4000)
        case(R, cfg, packed_input(R, cfg), "c3_fixture", [0, 256, 512, 514], a.threads)
    if "c3_seed1024" in a.cases:
        bench_input_case(R, a.threads)
    if "c2_newton" in a.cases:
        cfg = config(ref, 512, 3000, 3000)
        z = perturb(packed_input(R, cfg), 1e-3, np.random.default_rng(SEED + 2))
        newton_case(R, cfg, z, "c2_newton", a.threads, store_jacobian=True)
    if "c1_schemes" in a.cases:
        # C1 with the one- and three-stage Gauss-Legendre schemes (SchemeIRK 1, 3):
        # base shoot and the leading column of each field plus Delta
        for scheme in (1, 3):
            cfg = config(ref, 128, 1000, 1000)
            cfg["SchemeIRK"] = scheme
            case(R, cfg, packed_input(R, cfg), f"c1_scheme{scheme}", [0, 32, 64, 66], a.threads)
    if "c256_newton" in a.cases:
        # Ntau 256, 2000 + 2000 points: the Newton loop from a seeded 1e-3 perturbation
        cfg = config(ref, 256, 2000, 2000)
        z = perturb(packed_input(R, cfg), 1e-3, np.random.default_rng(SEED + 4))
        newton_case(R, cfg, z, "c256_newton", a.threads, store_jacobian=True)
    if "c2048" in a.cases:
        # Ntau 2048, the data file's 8000 + 8000 points: boundary data, RHS and
        # IRK steps, the base shoot and Jacobian columns 0..7 (one OpenMP round)
        cfg = config(ref, 2048, 8000, 8000)
        case(R, cfg, packed_input(R, cfg), "c2048", None, a.threads)
        d = dict(np.load(HERE / "ref_c2048.npz"))
        t = time.time()
        d["jac_idx"] = np.arange(8)
        d["jac_cols"] = R.jacobian_columns(cfg, d["in0"], d["out0"], 0, 8, a.threads)
        d["t_jac_s"] = time.time() - t
        np.savez_compressed(HERE / "ref_c2048.npz", **d)
        print("c2048 columns", d["jac_cols"].shape, f"{d['t_jac_s']:.0f} s")
    if "c3_newton" in a.cases:
        cfg = config(ref, 1024, 4000, 4000)
        z = perturb(packed_input(R, cfg), 1e-4, np.random.default_rng(SEED + 3))
        newton_case(R, cfg, z, "c3_newton", a.threads, store_jacobian=False)


if __name__ == "__main__":
    main()
