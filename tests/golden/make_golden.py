"""Generates the golden fixtures under tests/golden/ from the reference.

TEST INFRASTRUCTURE ONLY.  Run where the reference tree exists:

    python tests/golden/make_golden.py [--reference /root/reference]

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
"""
import argparse
import json
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args()
    ref = Path(a.reference)
    src = (ref / "test" / "test_init_gen.cpp").read_text()
    g = parse_init_gen(src)
    np.savez_compressed(HERE / "init_gen_128.npz", ntau=128, dim=4.0, delta=3.445501184653556, xl=0.001, xr=0.999,
                        **g)
    R = RefLib()
    rng = np.random.default_rng(SEED)
    # C1: Ntau=128, 1000+1000 points, full Jacobian and Newton step, fixture and seeded perturbation
    cfg = config(ref, 128, 1000, 1000)
    z = packed_input(R, cfg)
    case(R, cfg, z, "c1_fixture", range(96), a.threads, full_newton=True)
    zp = perturb(z, 1e-3, rng)
    case(R, cfg, zp, "c1_perturbed", range(96), a.threads, full_newton=True)
    newton_to_convergence(R, cfg, zp, "c1_newton", a.threads)
    # C2: Ntau=512, 3000+3000: base shoot and the leading column of each field plus Delta
    cfg = config(ref, 512, 3000, 3000)
    case(R, cfg, packed_input(R, cfg), "c2_fixture", [0, 128, 256, 258], a.threads)
    # C3: Ntau=1024, 4000+4000: the same columns (Up mode 1, psi_c mode 1, f_c DC, Delta)
    cfg = config(ref, 1024, 4000, 4000)
    case(R, cfg, packed_input(R, cfg), "c3_fixture", [0, 256, 512, 514], a.threads)


if __name__ == "__main__":
    main()
