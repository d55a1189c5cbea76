"""Failure parity of the dimension scan (bench.py's C4 section): the Newton
loops of three of its solves, on the engine and on the compiled reference.

TEST INFRASTRUCTURE ONLY.  Two steps:

    python tests/golden/make_c4_failure_golden.py --inputs      # on a GPU box
    python tests/golden/make_c4_failure_golden.py --reference   # where oracle/_ref is built

--inputs redraws bench.py's C4 solves exactly as its run_dscan does (seed
1028, the same re-draws; the engine resamples and packs the seed table) and
keeps solves 6, 14 and 15 (D = 3.85, 4.65, 4.69; Ntau 256 with 2000 points):
their SimulationConfig and initial unknowns -> ref_c4_failures.npz.
--reference runs the reference's Newton loop (NewtonSolver.cpp:279-366:
shoot, RMS mismatch, finite-difference J, dgesv, damped update) on each input
in a child process, because the reference ends the process (std::exit) when
an IRK sweep does not converge; each iteration's mismatch RMS is printed as
it is reached, and the last line says how the loop ended.  The histories are
added to the same file.
"""
import argparse
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
OUT = HERE / "ref_c4_failures.npz"
KEEP = (6, 14, 15)
CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from ref_lib import RefLib
cfg = json.loads(sys.argv[2])
x = np.array(json.loads(sys.argv[3]))
R = RefLib()
for it in range(cfg["MaxIterNewton"]):
    out = R.shoot(cfg, x)
    err = float(np.sqrt(np.mean(out ** 2)))
    print("err", repr(err), flush=True)
    if err < cfg["PrecisionNewton"]:
        print("end CONVERGED", flush=True)
        sys.exit(0)
    J = R.jacobian_columns(cfg, x, out, 0, x.size, 8)
    x = x + min(1.0, cfg["SlowError"] / err) * R.solve(J, -out)
print("end MAX_ITER", flush=True)
"""


def inputs():
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "parallel-critical-collapse_b200"))
    import bench
    import pcc

    eng = pcc.Engine(0)
    seeds = np.load(bench.SEEDS)
    rng = np.random.default_rng(1024 + 4)
    dims = 3.25 + 0.1 * np.arange(16)
    ns = rng.choice([128, 256, 512, 1024], 16)
    pts = [int(rng.choice([p for p in (2000, 4000, 6000, 8000) if p >= bench.MIN_POINTS[int(n)]])) for n in ns]
    kept = []
    for d, n, p in zip(dims, ns, pts):
        for _ in range(4):
            cfg, z = bench.seed_request(eng, seeds, d, int(n), int(p))
            z = bench.perturb(z, rng, 0.01)
            s = eng.solve(dict(cfg, PrecisionNewton=1e-30, MaxIterNewton=1000))
            try:
                s.shoot(z)
                s.close()
                kept.append((cfg, z))
                break
            except pcc.PccError:
                s.close()
    out = {}
    for i in KEEP:
        cfg, z = kept[i]
        out[f"cfg{i}"] = json.dumps(dict(cfg, PrecisionNewton=1e-10, MaxIterNewton=20))
        out[f"in0_{i}"] = z
    np.savez_compressed(OUT, keep=np.array(KEEP), **out)
    print("wrote", OUT)


def reference():
    d = dict(np.load(OUT))
    for i in KEEP:
        cfg = json.loads(str(d[f"cfg{i}"]))
        cfg.update({"Verbose": False, "Debug": False})
        r = subprocess.run([sys.executable, "-c", CHILD, str(HERE), json.dumps(cfg),
                            json.dumps(d[f"in0_{i}"].tolist())], capture_output=True, text=True, timeout=7200)
        errs = [float(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("err ")]
        ends = [l.split()[1] for l in r.stdout.splitlines() if l.startswith("end ")]
        end = ends[0] if ends else ("IRK_FAILED" if "No convergence" in (r.stdout + r.stderr) else f"exit {r.returncode}")
        d[f"ref_err{i}"] = np.array(errs)
        d[f"ref_end{i}"] = end
        print(i, cfg["Dim"], end, errs)
    np.savez_compressed(OUT, **d)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--inputs", action="store_true")
    ap.add_argument("--reference", action="store_true")
    a = ap.parse_args()
    if a.inputs:
        inputs()
    if a.reference:
        reference()
