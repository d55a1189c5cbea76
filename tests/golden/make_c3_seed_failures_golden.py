"""Failure parity of the benchmark's C3 free data: seeds that bench.py skips
because their base shoot does not converge, run through the compiled
reference's NewtonSolver::shoot.

TEST INFRASTRUCTURE ONLY.  Run where oracle/_ref is built:

    python tests/golden/make_c3_seed_failures_golden.py

For each seed, bench.workload(seed, 0.1) makes the input (the benchmark's
own construction); the reference's shoot runs in a child process because an
IRK step that does not converge ends the reference's process (std::exit,
ShootingSolver.cpp:78-80 on the left side, :121-123 on the right).  Its
message names the step's starting grid index i and the next one (i + 1
marching from x_L, i - 1 marching from x_R), which gives the side.  Output:
ref_c3_seed_failures.npz with the seeds, the inputs, and per seed the side
(0 left, 1 right, -1 converged) and the starting grid index.
"""
import json
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
SEEDS = (1025, 1026, 1027, 1028, 1029, 1030, 1031)  # 1031 converges: the control
CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from ref_lib import RefLib
cfg = json.loads(sys.argv[2])
x = np.array(json.loads(sys.argv[3]))
out = RefLib().shoot(cfg, x)
print("ok", float(np.sqrt(np.mean(out ** 2))), flush=True)
"""


def main():
    sys.path.insert(0, str(REPO))
    import bench

    inputs, sides, index = [], [], []
    for seed in SEEDS:
        cfg, in0 = bench.workload(seed, 0.1)
        r = subprocess.run([sys.executable, "-c", CHILD, str(HERE), json.dumps(cfg), json.dumps(in0.tolist())],
                           capture_output=True, text=True, timeout=1800)
        m = re.search(r"No convergence between grid point \S+ \((\d+)\)\s+and \S+ \((\d+)\)", r.stderr + r.stdout)
        if m:
            i, j = int(m.group(1)), int(m.group(2))
            sides.append(0 if j == i + 1 else 1)
            index.append(i)
        elif r.stdout.startswith("ok"):
            sides.append(-1)
            index.append(-1)
        else:
            raise RuntimeError(f"seed {seed}: {r.returncode} {r.stderr[-500:]}")
        inputs.append(in0)
        print(seed, "side", sides[-1], "grid index", index[-1], flush=True)
    cfg, _ = bench.workload(SEEDS[0], 0.1)
    np.savez_compressed(HERE / "ref_c3_seed_failures.npz", config=json.dumps(cfg), seeds=np.array(SEEDS),
                        in0=np.array(inputs), side=np.array(sides), grid_index=np.array(index), amp=0.1)


if __name__ == "__main__":
    main()
