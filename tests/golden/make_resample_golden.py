"""Golden vectors for spectral resampling: the reference's own
scripts/create_simulation_data.py `double` (imported from the reference tree)
applied to the Ntau = 128 near-solution fields of data/simulation_4D_128.json,
doubled three times (128 -> 256 -> 512 -> 1024).

Output: tests/golden/ref_resample_128.npz with the input fields and every
doubling.  Needs the reference tree: PCC_REFERENCE_ROOT=<checkout>.
"""
import importlib.util
import json
import pathlib

import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from ref_lib import reference_root  # noqa: E402


def main():
    REF = reference_root()
    spec = importlib.util.spec_from_file_location("create_simulation_data",
                                                  REF / "scripts" / "create_simulation_data.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    ic = json.loads((REF / "data" / "simulation_4D_128.json").read_text())["Initial_Conditions"]
    out = {}
    for name in ["fc", "psic", "Up"]:
        x = np.asarray(ic[name], dtype=np.float64)
        out[f"{name}_128"] = x
        for n in [256, 512, 1024]:
            x = np.asarray(mod.double(x.tolist()), dtype=np.float64)
            out[f"{name}_{n}"] = x
    np.savez_compressed(HERE / "ref_resample_128.npz", **out)
    print("wrote", HERE / "ref_resample_128.npz")


if __name__ == "__main__":
    main()
