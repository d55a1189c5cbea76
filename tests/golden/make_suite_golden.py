"""Golden fixtures for the dimension-continuation suite (the reference's
multiple-run mode, src/main.cpp:245-378): converged solutions at
five dimensions on each side of D = 4 in steps of 0.01 at the C1 resolution
(Ntau = 128, NLeft = NRight = 1000), produced by the reference's own
cc_openmp -m.

Two branches leave D = 4 (seeded with the reference's near-solution
data/simulation_4D_128.json): ascending 4.00 -> 4.04 (-r) and descending
4.00 -> 3.96.  Within a branch the reference seeds D_1, D_2 with the previous
converged solution and D_i (i >= 3) with a quadratic least-squares
extrapolation in D of the last three (main.cpp:279-354), so five dimensions
exercise every seeding rule.  Larger steps are out of reach of the
reference's damped Newton loop: with SlowError = 1e-3 the update is scaled by
1e-3/err, and from a seed 0.05 away in D the loop stalls and stops.

PrecisionNewton is 1e-12: the reference's default 1e-14 is below the residual
floor of this map (its Newton loop stalls near 1e-13 and then exits).

Output: tests/golden/ref_suite_128.npz with, per branch, the ordered dimension
keys, Delta, fc, psic, Up, Converged and IterNewton as the reference wrote them,
plus the suite input.  Needs oracle/_ref/cc_openmp (oracle/build_ref.sh) and the reference tree
(PCC_REFERENCE_ROOT=<checkout>, for data/simulation_4D_128.json).
"""
import json
import os
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent
CC = REPO / "oracle" / "_ref" / "cc_openmp"


def fixture_path():
    import sys

    sys.path.insert(0, str(HERE))
    from ref_lib import reference_root

    return reference_root() / "data" / "simulation_4D_128.json"
STEP = 0.01


def suite(dims, seed_cfg):
    out = {}
    for k, dim in enumerate(dims):
        c = dict(seed_cfg)
        c["Dim"] = float(dim)
        c["Converged"] = False
        if k == 0:
            c["Initial_Conditions"] = dict(seed_cfg["Initial_Conditions"])
        else:
            c["Initial_Conditions"] = {"Delta": None, "fc": None, "psic": None, "Up": None}
        out[f"{dim:.3f}"] = c
    return out


def main():
    base = json.loads(fixture_path().read_text())
    base.update({"NLeft": 1000, "NRight": 1000, "PrecisionNewton": 1e-12, "MaxIterNewton": 20,
                 "Verbose": False, "Debug": False})
    up = [4.0 + STEP * i for i in range(5)]         # 4.00 .. 4.04
    down = [4.0 - STEP * i for i in range(5)]       # 4.00 .. 3.96
    result = {}
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
    with tempfile.TemporaryDirectory() as tmp:
        for name, dims, flags in [("up", up, ["-r"]), ("down", down, [])]:
            path = pathlib.Path(tmp) / f"suite_{name}.json"
            path.write_text(json.dumps(suite(dims, base)))
            r = subprocess.run([str(CC), "-m", *flags, "-i", str(path)], capture_output=True, text=True,
                               env=env, cwd=tmp)
            sys.stdout.write("\n".join(l for l in r.stdout.splitlines()
                                        if l.startswith(("Starting simulation", "Mismatch norm", "The solution")))
                             + "\n")
            if r.returncode != 0:
                sys.stderr.write(r.stderr[-2000:])
                raise SystemExit(f"cc_openmp -m failed on branch {name}")
            res = json.loads(path.read_text())
            keys = [f"{d:.3f}" for d in dims]
            result[f"{name}_keys"] = np.array(keys)
            result[f"{name}_delta"] = np.array([res[k]["Initial_Conditions"]["Delta"] for k in keys])
            for f in ["fc", "psic", "Up"]:
                result[f"{name}_{f}"] = np.array([res[k]["Initial_Conditions"][f] for k in keys])
            result[f"{name}_converged"] = np.array([bool(res[k]["Converged"]) for k in keys])
            result[f"{name}_iters"] = np.array([int(res[k].get("IterNewton", -1)) for k in keys])
    result["config"] = json.dumps({k: v for k, v in base.items() if k != "Initial_Conditions"})
    result["seed_ic"] = json.dumps(base["Initial_Conditions"])
    np.savez_compressed(HERE / "ref_suite_128.npz", **result)
    print("wrote", HERE / "ref_suite_128.npz")


if __name__ == "__main__":
    main()
