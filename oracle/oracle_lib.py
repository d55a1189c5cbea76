"""ctypes wrapper of the C oracle (oracle/pcc_oracle.c -> oracle/libpcc_oracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the cpu_baseline
leg of bench.py may load this module, as the checker; the product never does.
"""
import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "pcc_oracle.c"
SO = HERE / "libpcc_oracle.so"

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_LL = ctypes.POINTER(ctypes.c_longlong)


class OrcCfg(ctypes.Structure):
    _fields_ = [
        ("ntau", ctypes.c_int),
        ("dim", ctypes.c_double),
        ("xl", ctypes.c_double),
        ("xm", ctypes.c_double),
        ("xr", ctypes.c_double),
        ("eps_newton", ctypes.c_double),
        ("nl", ctypes.c_int),
        ("nr", ctypes.c_int),
        ("prec_irk", ctypes.c_double),
        ("scheme", ctypes.c_int),
        ("max_irk", ctypes.c_int),
    ]


def cfg_from_json(cfg):
    """Builds the oracle config from a reference SimulationConfig dict."""
    return OrcCfg(int(cfg["Ntau"]), float(cfg["Dim"]), float(cfg["XLeft"]), float(cfg["XMid"]),
                  float(cfg["XRight"]), float(cfg["EpsNewton"]), int(cfg["NLeft"]), int(cfg["NRight"]),
                  float(cfg["PrecisionIRK"]), int(cfg["SchemeIRK"]), int(cfg["MaxIterIRK"]))


def build(force=False):
    """Compiles the oracle (gcc, -O2, no fast-math)."""
    if SO.exists() and not force and SO.stat().st_mtime >= SRC.stat().st_mtime:
        return SO
    cmd = ["gcc", "-std=c99", "-O2", "-march=x86-64-v3", "-fPIC", "-shared", "-o", str(SO), str(SRC), "-lm"]
    subprocess.run(cmd, check=True)
    return SO


def _p(a):
    return a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    def __init__(self, path=None):
        path = Path(path) if path else SO
        if not path.exists():
            build()
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        ci, cd = ctypes.c_int, ctypes.c_double
        L.orc_rms.restype = cd
        L.orc_rms.argtypes = [ci, _D]
        L.orc_irk_step.argtypes = [ci, cd, ci, cd, ci, _D, cd, cd, _D, _I]
        L.orc_rhs.argtypes = [ci, cd, _D, cd, _D]
        L.orc_left_expansion.argtypes = [ci, cd, cd, _D, _D, cd, _D]
        L.orc_right_expansion.argtypes = [ci, cd, cd, _D, cd, _D]
        L.orc_pack.argtypes = [ci, _D, _D, _D, _D]
        L.orc_unpack.argtypes = [ci, _D, _D, _D, _D]
        L.orc_state_to_fields.argtypes = [ci, cd, _D, cd] + [_D] * 7
        L.orc_state_to_fields_light.argtypes = [ci, _D, _D, _D, _D]
        L.orc_fields_to_state.argtypes = [ci, _D, _D, _D, _D]
        L.orc_grid.argtypes = [ctypes.POINTER(OrcCfg), _D]
        L.orc_sweep.argtypes = [ctypes.POINTER(OrcCfg), _D, ci, ci, ci, _D, _D, _I, _LL]
        L.orc_shoot.argtypes = [ctypes.POINTER(OrcCfg), _D, _D, _D, _LL]
        L.orc_jacobian_columns.argtypes = [ctypes.POINTER(OrcCfg), _D, _D, _D, ci, ci, _D, _LL]
        L.orc_dgesv.argtypes = [ci, _D, _D]
        L.orc_solve_inhom.argtypes = [ci, _D, _D, _D, cd]
        L.orc_forward_real.argtypes = [ci, _D, _D]
        L.orc_backward_real.argtypes = [ci, _D, _D]
        L.orc_dft.argtypes = [ci, _D, ci]

    def pack(self, n, up, psic, fc):
        z = np.zeros(3 * n // 4)
        a, b, c = _f64(up), _f64(psic), _f64(fc)
        self.lib.orc_pack(n, _p(a), _p(b), _p(c), _p(z))
        return z

    def unpack(self, n, z):
        z = _f64(z)
        a, b, c = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.orc_unpack(n, _p(z), _p(a), _p(b), _p(c))
        return a, b, c

    def left_expansion(self, n, dim, xl, fc, psic, delta):
        y = np.zeros(n)
        f, p = _f64(fc), _f64(psic)
        self.lib.orc_left_expansion(n, dim, xl, _p(f), _p(p), delta, _p(y))
        return y

    def right_expansion(self, n, dim, xr, up, delta):
        y = np.zeros(n)
        u = _f64(up)
        self.lib.orc_right_expansion(n, dim, xr, _p(u), delta, _p(y))
        return y

    def state_to_fields(self, n, dim, y, x):
        y = _f64(y)
        outs = [np.zeros(n) for _ in range(7)]
        self.lib.orc_state_to_fields(n, dim, _p(y), x, *[_p(o) for o in outs])
        return dict(zip(["U", "V", "F", "IA2", "dUdt", "dVdt", "dFdt"], outs))

    def state_to_fields_light(self, n, y):
        y = _f64(y)
        u, v, f = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.orc_state_to_fields_light(n, _p(y), _p(u), _p(v), _p(f))
        return u, v, f

    def rhs(self, n, dim, y, x):
        y = _f64(y)
        d = np.zeros(n)
        self.lib.orc_rhs(n, dim, _p(y), x, _p(d))
        return d

    def irk_step(self, n, dim, scheme, precision, max_its, y, x_in, x_out):
        y = _f64(y)
        out = np.zeros(n)
        its = ctypes.c_int(0)
        conv = self.lib.orc_irk_step(n, dim, scheme, precision, max_its, _p(y), x_in, x_out, _p(out),
                                     ctypes.byref(its))
        return out, its.value, bool(conv)

    def grid(self, cfg):
        c = cfg_from_json(cfg)
        g = np.zeros(c.nl + c.nr + 1)
        self.lib.orc_grid(ctypes.byref(c), _p(g))
        return g

    def sweep(self, cfg, y_init, forward, grid=None):
        c = cfg_from_json(cfg)
        g = self.grid(cfg) if grid is None else _f64(grid)
        y = _f64(y_init)
        out = np.zeros(c.ntau)
        fail = ctypes.c_int(-1)
        ev = ctypes.c_longlong(0)
        if forward:
            st = self.lib.orc_sweep(ctypes.byref(c), _p(g), 0, c.nl, 1, _p(y), _p(out), ctypes.byref(fail),
                                    ctypes.byref(ev))
        else:
            st = self.lib.orc_sweep(ctypes.byref(c), _p(g), c.nl + c.nr, c.nl, 0, _p(y), _p(out),
                                    ctypes.byref(fail), ctypes.byref(ev))
        return out, st, fail.value, ev.value

    def shoot(self, cfg, in0, grid=None):
        c = cfg_from_json(cfg)
        g = self.grid(cfg) if grid is None else _f64(grid)
        in0 = _f64(in0)
        out = np.zeros_like(in0)
        ev = ctypes.c_longlong(0)
        st = self.lib.orc_shoot(ctypes.byref(c), _p(g), _p(in0), _p(out), ctypes.byref(ev))
        return out, st, ev.value

    def jacobian_columns(self, cfg, in0, out0, c0, c1, grid=None):
        c = cfg_from_json(cfg)
        g = self.grid(cfg) if grid is None else _f64(grid)
        in0, out0 = _f64(in0), _f64(out0)
        cols = np.zeros((c1 - c0, in0.size))
        ev = ctypes.c_longlong(0)
        st = self.lib.orc_jacobian_columns(ctypes.byref(c), _p(g), _p(in0), _p(out0), c0, c1, _p(cols),
                                           ctypes.byref(ev))
        return cols.T.copy(), st, ev.value

    def dgesv(self, a, b):
        a = _f64(a).copy()
        b = _f64(b).copy()
        st = self.lib.orc_dgesv(b.size, _p(a), _p(b))
        return b, st

    def rms(self, v):
        v = _f64(v)
        return self.lib.orc_rms(v.size, _p(v))
