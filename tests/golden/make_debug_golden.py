"""Golden Debug output of the reference: cc_openmp -s on the C1 setup
(data/simulation_4D_128.json with NLeft = NRight = 1000) with Debug on
(DebugNx = 100, DebugNtau = 4) and one Newton iteration.  The reference then
writes fields_<D>_0.json (ShootingSolver.cpp:85-97, 128-138, the base shoot's
field snapshots) and jacobian_<D>_1.csv (NewtonSolver.cpp:337-341) next to the
input and exits (one iteration cannot meet PrecisionNewton = 1e-30).

Output: tests/golden/ref_debug_128.npz: the snapshot keys (std::to_string of
x), the A/U/V/f arrays per key, the Jacobian, and the input configuration.
Needs oracle/_ref/cc_openmp (oracle/build_ref.sh) and the reference tree
(PCC_REFERENCE_ROOT=<checkout>, for data/simulation_4D_128.json).
"""
import json
import os
import pathlib
import subprocess
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


def main():
    cfg = json.loads(fixture_path().read_text())
    cfg.update({"NLeft": 1000, "NRight": 1000, "PrecisionNewton": 1e-30, "MaxIterNewton": 1, "Verbose": False,
                "Debug": True, "DebugNx": 100, "DebugNtau": 4, "Converged": False})
    with tempfile.TemporaryDirectory() as tmp:
        path = pathlib.Path(tmp) / "sim.json"
        path.write_text(json.dumps(cfg))
        env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
        r = subprocess.run([str(CC), "-s", "-i", str(path)], capture_output=True, text=True, env=env, cwd=tmp)
        files = sorted(p.name for p in pathlib.Path(tmp).iterdir())
        print(r.returncode, files)
        fj = [f for f in files if f.startswith("fields_")]
        jc = [f for f in files if f.startswith("jacobian_")]
        assert len(fj) == 1 and len(jc) == 1, files
        fields = json.loads((pathlib.Path(tmp) / fj[0]).read_text())
        J = np.loadtxt(pathlib.Path(tmp) / jc[0], delimiter=",")
    keys = list(fields.keys())
    out = {"keys": np.array(keys), "fields_file": fj[0], "jacobian_file": jc[0], "J": J,
           "config": json.dumps(cfg)}
    for q in ["A", "U", "V", "f"]:
        out[q] = np.array([fields[k][q] for k in keys])
    np.savez_compressed(HERE / "ref_debug_128.npz", **out)
    print("wrote", HERE / "ref_debug_128.npz", len(keys), "snapshots, J", J.shape)


if __name__ == "__main__":
    main()
