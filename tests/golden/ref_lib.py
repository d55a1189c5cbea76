"""ctypes view of the compiled reference (oracle/_ref/libpcc_ref.so).

TEST INFRASTRUCTURE ONLY: used by make_golden.py (fixture generation, in the
container that holds the reference tree) and by the CPU reference arm of
bench.py.  The library is built by oracle/build_ref.sh from the reference's own
sources; see oracle/ref_harness.cpp for the entry points.
"""
import ctypes
import json
import os
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
REF_SO = REPO / "oracle" / "_ref" / "libpcc_ref.so"

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _p(a):
    return a.ctypes.data_as(_D)


class RefLib:
    def __init__(self, path=REF_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh")
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        c_int, c_double, c_char_p = ctypes.c_int, ctypes.c_double, ctypes.c_char_p
        L.ref_pack.argtypes = [c_int, c_double, c_double, _D, _D, _D, _D]
        L.ref_unpack.argtypes = [c_int, c_double, c_double, _D, _D, _D, _D]
        L.ref_left_expansion.argtypes = [c_int, c_double, c_double, _D, _D, c_double, _D]
        L.ref_right_expansion.argtypes = [c_int, c_double, c_double, _D, c_double, _D]
        L.ref_state_to_fields.argtypes = [c_int, c_double, _D, c_double] + [_D] * 7
        L.ref_rhs.argtypes = [c_int, c_double, _D, c_double, _D]
        L.ref_irk_step.argtypes = [c_int, c_double, c_int, c_double, c_int, _D, c_double, c_double, _D, _I, _I]
        L.ref_sweep.argtypes = [c_char_p, _D, c_int, _D]
        L.ref_grid.argtypes = [c_char_p, _D]
        L.ref_shoot.argtypes = [c_char_p, _D, _D]
        L.ref_jacobian_columns.argtypes = [c_char_p, _D, _D, c_int, c_int, _D, c_int]
        L.ref_solve.argtypes = [c_int, _D, _D, _D]

    # -- spectral packing -------------------------------------------------
    def pack(self, ntau, dim, delta, up, psic, fc):
        z = np.zeros(3 * ntau // 4)
        a, b, c = (np.ascontiguousarray(x, dtype=np.float64) for x in (up, psic, fc))
        self.lib.ref_pack(ntau, dim, delta, _p(a), _p(b), _p(c), _p(z))
        return z

    def unpack(self, ntau, dim, delta, z):
        z = np.ascontiguousarray(z, dtype=np.float64)
        up, psic, fc = np.zeros(ntau), np.zeros(ntau), np.zeros(ntau)
        self.lib.ref_unpack(ntau, dim, delta, _p(z), _p(up), _p(psic), _p(fc))
        return up, psic, fc

    def left_expansion(self, ntau, dim, xl, fc, psic, delta):
        y = np.zeros(ntau)
        f, p = (np.ascontiguousarray(x, dtype=np.float64) for x in (fc, psic))
        self.lib.ref_left_expansion(ntau, dim, xl, _p(f), _p(p), delta, _p(y))
        return y

    def right_expansion(self, ntau, dim, xr, up, delta):
        y = np.zeros(ntau)
        u = np.ascontiguousarray(up, dtype=np.float64)
        self.lib.ref_right_expansion(ntau, dim, xr, _p(u), delta, _p(y))
        return y

    # -- state / RHS / IRK ------------------------------------------------
    def state_to_fields(self, ntau, dim, y, x):
        y = np.ascontiguousarray(y, dtype=np.float64)
        outs = [np.zeros(ntau) for _ in range(7)]
        self.lib.ref_state_to_fields(ntau, dim, _p(y), x, *[_p(o) for o in outs])
        return dict(zip(["U", "V", "F", "IA2", "dUdt", "dVdt", "dFdt"], outs))

    def rhs(self, ntau, dim, y, x):
        y = np.ascontiguousarray(y, dtype=np.float64)
        dy = np.zeros(ntau)
        self.lib.ref_rhs(ntau, dim, _p(y), x, _p(dy))
        return dy

    def irk_step(self, ntau, dim, scheme, precision, max_its, y, x_in, x_out):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(ntau)
        its, conv = ctypes.c_int(0), ctypes.c_int(0)
        self.lib.ref_irk_step(ntau, dim, scheme, precision, max_its, _p(y), x_in, x_out, _p(out),
                              ctypes.byref(its), ctypes.byref(conv))
        return out, its.value, bool(conv.value)

    # -- shooting / Newton --------------------------------------------------
    def grid(self, cfg):
        g = np.zeros(cfg["NLeft"] + cfg["NRight"] + 1)
        self.lib.ref_grid(json.dumps(cfg).encode(), _p(g))
        return g

    def sweep(self, cfg, y_init, forward):
        y = np.ascontiguousarray(y_init, dtype=np.float64)
        out = np.zeros(cfg["Ntau"])
        self.lib.ref_sweep(json.dumps(cfg).encode(), _p(y), 1 if forward else 0, _p(out))
        return out

    def shoot(self, cfg, in0):
        in0 = np.ascontiguousarray(in0, dtype=np.float64)
        out = np.zeros_like(in0)
        self.lib.ref_shoot(json.dumps(cfg).encode(), _p(in0), _p(out))
        return out

    def jacobian_columns(self, cfg, in0, out0, c0, c1, nthreads=0):
        in0 = np.ascontiguousarray(in0, dtype=np.float64)
        out0 = np.ascontiguousarray(out0, dtype=np.float64)
        cols = np.zeros((c1 - c0, in0.size))
        self.lib.ref_jacobian_columns(json.dumps(cfg).encode(), _p(in0), _p(out0), c0, c1, _p(cols),
                                      int(nthreads))
        return cols.T.copy()  # rows x (c1-c0)

    def solve(self, a, rhs):
        a = np.ascontiguousarray(a, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs)
        self.lib.ref_solve(rhs.size, _p(a), _p(rhs), _p(x))
        return x


def available():
    return REF_SO.exists()


def reference_root():
    """The reference checkout the fixture scripts read (data/, test/, scripts/):
    $PCC_REFERENCE_ROOT, which they require."""
    root = os.environ.get("PCC_REFERENCE_ROOT")
    if not root or not Path(root, "src").is_dir():
        raise SystemExit("set PCC_REFERENCE_ROOT to the reference checkout (the directory holding src/ and data/)")
    return Path(root)
