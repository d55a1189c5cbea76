"""Converged starting data for the dimension-scan and serving workloads of
bench.py: solutions at D = 3.25 .. 4.75 in steps of 0.01 (Ntau = 128,
NLeft = NRight = 1000), computed by this engine's dimension continuation
(cc_b200 -m, the reference's multiple-run mode) from the converged D = 4
solution of tests/golden/ref_c1_newton.npz, the two branches in lockstep.

Run on a GPU box:  python bench_data/make_dscan_seeds.py [--extend-to 4.75]
Output: bench_data/dscan_seeds_128.npz (keys D, delta, fc, psic, Up, err,
converged) and the two suite files it came from, under a temporary folder.
--extend-to D continues the ascending branch of an existing table past its
largest dimension in steps of --step (default 0.005), seeded with the table's
last three converged dimensions as the reference's suite mode seeds a new
dimension, and merges the converged ones into the table.
The reference's damped Newton loop needs the small step (from 0.05 away it
stalls, see tests/golden/make_suite_golden.py).  PrecisionNewton is 1e-10:
away from D = 4 the mismatch floor of this map rises above 1e-12 (2e-12 at
D = 4.19).  A branch that fails stops there; the table holds every converged
dimension.
"""
import json
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO / "parallel-critical-collapse_b200"))

STEP = 0.01


def main():
    import pcc

    d = np.load(REPO / "tests" / "golden" / "ref_c1_newton.npz")
    cfg = json.loads(str(d["config"]))
    cfg.update({"PrecisionNewton": 1e-10, "MaxIterNewton": 40, "Verbose": False, "Debug": False})
    x = d["x_star"].copy()
    nn = x.size
    delta = float(x[2 * nn // 3 + 2])
    x[2 * nn // 3 + 2] = 0.0
    eng = pcc.Engine(0)
    up_f, ps_f, fc_f = eng.unpack(cfg["Ntau"], x)
    eng.close()
    seed = {"Delta": delta, "fc": fc_f.tolist(), "psic": ps_f.tolist(), "Up": up_f.tolist()}
    n_steps = int(round(0.75 / STEP))
    branches = {"up": [4.0 + STEP * i for i in range(n_steps + 1)],
                "down": [4.0 - STEP * i for i in range(n_steps + 1)]}
    res = {}
    with tempfile.TemporaryDirectory() as tmp:
        paths = {}
        for name, dims in branches.items():
            suite = {}
            for k, dim in enumerate(dims):
                c = dict(cfg)
                c["Dim"] = round(dim, 4)
                c["Converged"] = False
                c["Initial_Conditions"] = seed if k == 0 else {"Delta": None, "fc": None, "psic": None, "Up": None}
                suite[f"{dim:.3f}"] = c
            paths[name] = pathlib.Path(tmp) / f"{name}.json"
            paths[name].write_text(json.dumps(suite))
        r = subprocess.run([str(REPO / "parallel-critical-collapse_b200" / "cc_b200"), "-m",
                            "--suite", str(paths["up"]), "asc", "--suite", str(paths["down"]), "desc"],
                           capture_output=True, text=True)
        print("\n".join(l for l in r.stdout.splitlines() if l.startswith("D = ")))
        print(r.stderr[-1500:])
        for name in branches:
            res.update(json.loads(paths[name].read_text()))
    keys = sorted((k for k, v in res.items() if v.get("Converged") and v["Initial_Conditions"]["fc"]), key=float)
    out = {
        "D": np.array([float(k) for k in keys]),
        "delta": np.array([res[k]["Initial_Conditions"]["Delta"] for k in keys]),
        "err": np.array([res[k].get("mismatchNorm", np.nan) for k in keys]),
        "config": json.dumps({k: v for k, v in cfg.items() if k != "Initial_Conditions"}),
    }
    for f in ["fc", "psic", "Up"]:
        out[f] = np.array([res[k]["Initial_Conditions"][f] for k in keys])
    np.savez_compressed(HERE / "dscan_seeds_128.npz", **out)
    print(f"{len(keys)} converged dimensions from {out['D'].min()} to {out['D'].max()}")


def extend(d_max, step, prec):
    """Continues the ascending branch of the table to d_max."""
    t = dict(np.load(HERE / "dscan_seeds_128.npz"))
    cfg = json.loads(str(t["config"]))
    cfg.update({"PrecisionNewton": prec, "MaxIterNewton": 60, "Verbose": False, "Debug": False})
    order = np.argsort(t["D"])
    suite = {}
    for i in order[-3:]:
        c = dict(cfg)
        c["Dim"] = float(t["D"][i])
        c["Converged"] = True
        c["Initial_Conditions"] = {"Delta": float(t["delta"][i]), "fc": t["fc"][i].tolist(),
                                   "psic": t["psic"][i].tolist(), "Up": t["Up"][i].tolist()}
        suite[f"{t['D'][i]:.3f}"] = c
    d = float(t["D"][order[-1]])
    new_keys = []
    while d + step <= d_max + 1e-9:
        d = round(d + step, 4)
        c = dict(cfg)
        c["Dim"] = d
        c["Converged"] = False
        c["Initial_Conditions"] = {"Delta": None, "fc": None, "psic": None, "Up": None}
        suite[f"{d:.3f}"] = c
        new_keys.append(f"{d:.3f}")
    with tempfile.TemporaryDirectory() as tmp:
        path = pathlib.Path(tmp) / "ext.json"
        path.write_text(json.dumps(suite))
        r = subprocess.run([str(REPO / "parallel-critical-collapse_b200" / "cc_b200"), "-m", "--suite", str(path),
                            "asc"], capture_output=True, text=True)
        print("\n".join(l for l in r.stdout.splitlines() if l.startswith("D = ")))
        print(r.stderr[-1500:])
        res = json.loads(path.read_text())
    got = [k for k in new_keys if res[k].get("Converged") and res[k]["Initial_Conditions"]["fc"]]
    if not got:
        print("no new dimension converged")
        return
    D = np.concatenate([t["D"], [float(k) for k in got]])
    idx = np.argsort(D)
    out = {"D": D[idx], "config": t["config"],
           "delta": np.concatenate([t["delta"], [res[k]["Initial_Conditions"]["Delta"] for k in got]])[idx],
           "err": np.concatenate([t["err"], [res[k].get("mismatchNorm", np.nan) for k in got]])[idx]}
    for f in ["fc", "psic", "Up"]:
        out[f] = np.concatenate([t[f], np.array([res[k]["Initial_Conditions"][f] for k in got])])[idx]
    np.savez_compressed(HERE / "dscan_seeds_128.npz", **out)
    print(f"added {len(got)} dimensions up to {max(float(k) for k in got)}")


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--extend-to", type=float, default=0.0)
    ap.add_argument("--step", type=float, default=0.005)
    ap.add_argument("--precision", type=float, default=1e-10)
    a = ap.parse_args()
    if a.extend_to:
        extend(a.extend_to, a.step, a.precision)
    else:
        main()
