"""ctypes binding of include/pcc.h (libpcc_b200.so).

This is how Python callers (the tests, bench.py, a ctypes-based driver) reach
the CUDA engine.  It loads the in-tree library and raises if it is missing:
there is no CPU fallback.

    from pcc import Engine, SolveDesc
    eng = Engine(device=0)
    solve = eng.solve(SolveDesc.from_config(cfg_dict))
    out0 = solve.shoot(in0)
    J = solve.jacobian(in0, out0)
"""
import ctypes
import json
import os
import weakref
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpcc_b200.so"

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)

STATUS = ["PCC_OK", "PCC_ERR_INVALID_ARG", "PCC_ERR_CUDA", "PCC_ERR_OOM", "PCC_ERR_IRK_NO_CONVERGENCE",
          "PCC_ERR_DELTA_MISMATCH", "PCC_ERR_NAN", "PCC_ERR_LU_SINGULAR", "PCC_ERR_IR_STALL", "PCC_ERR_UNSUPPORTED",
          "PCC_ERR_NEWTON_NO_CONVERGENCE", "PCC_ERR_BUSY", "PCC_ERR_TIMEOUT"]
PREC_FP64, PREC_MIXED = 0, 1
PCC_ERR_INVALID_ARG, PCC_ERR_NAN, PCC_ERR_BUSY, PCC_ERR_TIMEOUT = 1, 6, 11, 12

# every function include/pcc.h declares
EXPORTS = ["pcc_ctx_create", "pcc_ctx_destroy", "pcc_status_string", "pcc_last_error", "pcc_solve_create",
           "pcc_solve_destroy", "pcc_solve_grid", "pcc_shoot", "pcc_jacobian", "pcc_jacobian_device",
           "pcc_solve_sync", "pcc_jacobian_columns", "pcc_lu_solve", "pcc_newton_step", "pcc_rhs_eval",
           "pcc_irk_step", "pcc_boundary_data", "pcc_sweep", "pcc_fp64_peak", "pcc_pack_fields",
           "pcc_unpack_fields", "pcc_expansions", "pcc_solve_set_grid", "pcc_dft", "pcc_expansions_static",
           "pcc_jacobian_batch", "pcc_newton_begin", "pcc_newton_iterate", "pcc_newton_result",
           "pcc_newton_solve", "pcc_serve_start", "pcc_submit", "pcc_poll", "pcc_wait", "pcc_serve_stats",
           "pcc_serve_stop", "pcc_resample_fields", "pcc_shoot_debug", "pcc_jacobian_columns_device",
           "pcc_march_tuning", "pcc_sweep_plan"]

NEWTON_CODES = ["RUNNING", "CONVERGED", "STOPPED", "MAX_ITER", "IRK_FAILED", "DELTA_MISMATCH", "SINGULAR"]


class PccError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        self.name = STATUS[status] if 0 <= status < len(STATUS) else str(status)
        super().__init__(f"{self.name}: {msg}")


class SolveDesc(ctypes.Structure):
    _fields_ = [("ntau", ctypes.c_int), ("dim", ctypes.c_double), ("xl", ctypes.c_double),
                ("xm", ctypes.c_double), ("xr", ctypes.c_double), ("eps_newton", ctypes.c_double),
                ("nl", ctypes.c_int), ("nr", ctypes.c_int), ("prec_irk", ctypes.c_double),
                ("scheme", ctypes.c_int), ("max_irk", ctypes.c_int), ("prec_newton", ctypes.c_double),
                ("slow_error", ctypes.c_double), ("max_newton", ctypes.c_int), ("irk_predictor", ctypes.c_int),
                ("shoot_both_sides", ctypes.c_int)]

    @classmethod
    def from_config(cls, cfg):
        """From a reference SimulationConfig dict (include/SimulationConfig.hpp:73-137)."""
        return cls(int(cfg["Ntau"]), float(cfg["Dim"]), float(cfg["XLeft"]), float(cfg["XMid"]),
                   float(cfg["XRight"]), float(cfg["EpsNewton"]), int(cfg["NLeft"]), int(cfg["NRight"]),
                   float(cfg["PrecisionIRK"]), int(cfg["SchemeIRK"]), int(cfg["MaxIterIRK"]),
                   float(cfg.get("PrecisionNewton", 1e-14)), float(cfg.get("SlowError", 1e-3)),
                   int(cfg.get("MaxIterNewton", 100)), int(bool(cfg.get("IRKPredictor", False))),
                   int(bool(cfg.get("ShootBothSides", False))))


class Stats(ctypes.Structure):
    _fields_ = [("rhs_evals", ctypes.c_longlong), ("irk_iterations", ctypes.c_longlong),
                ("irk_steps", ctypes.c_longlong), ("shoots", ctypes.c_longlong), ("ms_prologue", ctypes.c_double),
                ("ms_sweep", ctypes.c_double), ("ms_epilogue", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("fail_column", ctypes.c_int), ("fail_side", ctypes.c_int), ("fail_grid_index", ctypes.c_int),
                ("sweep_ctas", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RefineReport(ctypes.Structure):
    _fields_ = [("rel_err_vs_fp64", ctypes.c_double), ("residual_norm", ctypes.c_double),
                ("refinement_steps", ctypes.c_int), ("fell_back_to_fp64", ctypes.c_int), ("ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NewtonState(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("code", ctypes.c_int), ("err", ctypes.c_double),
                ("err_old", ctypes.c_double), ("fail_column", ctypes.c_int), ("fail_side", ctypes.c_int),
                ("fail_grid_index", ctypes.c_int), ("lu_refinement_steps", ctypes.c_int),
                ("lu_fell_back", ctypes.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["state"] = NEWTON_CODES[self.code] if 0 <= self.code < len(NEWTON_CODES) else str(self.code)
        return d


class ServeOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_active", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("desc", SolveDesc), ("in0", _D), ("precision", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("done", ctypes.c_int), ("status", ctypes.c_int), ("newton", NewtonState),
                ("ms_queued", ctypes.c_double), ("ms_latency", ctypes.c_double),
                ("footprint_bytes", ctypes.c_size_t)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "newton"}
        d["newton"] = self.newton.as_dict()
        d["status_name"] = STATUS[self.status] if 0 <= self.status < len(STATUS) else str(self.status)
        return d


class ServeInfo(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("launches", ctypes.c_longlong), ("sweeps", ctypes.c_longlong), ("active", ctypes.c_int),
                ("waiting", ctypes.c_int), ("bytes_in_use", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path=None):
    """Loads libpcc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run parallel-critical-collapse_b200/build.py")
    L = ctypes.CDLL(str(p))
    vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.pcc_status_string.restype = ctypes.c_char_p
    L.pcc_status_string.argtypes = [ci]
    L.pcc_last_error.restype = ctypes.c_char_p
    L.pcc_last_error.argtypes = [vp]
    L.pcc_ctx_create.argtypes = [ci, vp, ctypes.POINTER(vp)]
    L.pcc_ctx_destroy.argtypes = [vp]
    L.pcc_solve_create.argtypes = [vp, ctypes.POINTER(SolveDesc), ctypes.POINTER(vp)]
    L.pcc_solve_destroy.argtypes = [vp]
    L.pcc_solve_grid.argtypes = [vp, _D]
    L.pcc_shoot.argtypes = [vp, _D, _D, ctypes.POINTER(Stats)]
    L.pcc_jacobian.argtypes = [vp, _D, _D, _D, ctypes.POINTER(Stats)]
    L.pcc_jacobian_device.argtypes = [vp, vp, vp, vp]
    L.pcc_solve_sync.argtypes = [vp, ctypes.POINTER(Stats)]
    L.pcc_jacobian_columns.argtypes = [vp, _D, _D, ci, ci, _D, ctypes.POINTER(Stats)]
    L.pcc_lu_solve.argtypes = [vp, ci, _D, _D, _D, ci, ctypes.POINTER(RefineReport)]
    L.pcc_newton_step.argtypes = [vp, _D, _D, ci, ctypes.POINTER(Stats), ctypes.POINTER(RefineReport)]
    L.pcc_rhs_eval.argtypes = [vp, ci, cd, ci, _D, _D, _D]
    L.pcc_irk_step.argtypes = [vp, ci, cd, ci, cd, ci, ci, _D, _D, _D, _D, _I]
    L.pcc_boundary_data.argtypes = [vp, _D, _D, _D]
    L.pcc_sweep.argtypes = [vp, ci, _I, _D, _D, ctypes.POINTER(Stats)]
    L.pcc_fp64_peak.argtypes = [vp, ctypes.POINTER(cd)]
    L.pcc_pack_fields.argtypes = [vp, ci, _D, _D, _D, _D]
    L.pcc_unpack_fields.argtypes = [vp, ci, _D, _D, _D, _D]
    L.pcc_expansions.argtypes = [vp, ci, cd, cd, cd, cd, _D, _D, _D, _D, _D]
    L.pcc_solve_set_grid.argtypes = [vp, _D]
    L.pcc_dft.argtypes = [vp, ci, ci, ci, _D, _D]
    L.pcc_expansions_static.argtypes = [vp, ci, cd, cd, cd, cd, vp, vp, vp, vp, vp]
    PP = ctypes.POINTER(vp)
    L.pcc_jacobian_batch.argtypes = [vp, ci, PP, PP, PP, PP, ctypes.POINTER(Stats)]
    L.pcc_newton_begin.argtypes = [vp, _D]
    L.pcc_newton_iterate.argtypes = [vp, ci, PP, ci, ctypes.POINTER(NewtonState), ctypes.POINTER(Stats)]
    L.pcc_newton_result.argtypes = [vp, _D, ctypes.POINTER(NewtonState)]
    L.pcc_newton_solve.argtypes = [vp, ci, PP, PP, ci, ctypes.POINTER(NewtonState), ctypes.POINTER(Stats)]
    L.pcc_serve_start.argtypes = [vp, ctypes.POINTER(ServeOpts)]
    L.pcc_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]
    L.pcc_poll.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(Result), _D]
    L.pcc_wait.argtypes = [vp, ctypes.c_uint64, cd, ctypes.POINTER(Result), _D]
    L.pcc_serve_stats.argtypes = [vp, ctypes.POINTER(ServeInfo)]
    L.pcc_serve_stop.argtypes = [vp]
    L.pcc_resample_fields.argtypes = [vp, ci, ci, ci, _D, _D]
    L.pcc_shoot_debug.argtypes = [vp, _D, _D, ci, ci, _I, _I, _D, ctypes.POINTER(Stats)]
    L.pcc_jacobian_columns_device.argtypes = [vp, vp, vp, ci, ci, vp]
    L.pcc_march_tuning.argtypes = [vp, ci, ci, _I, _D, _D]
    L.pcc_sweep_plan.argtypes = [ci, ci, ci, ci, _I, ci]
    for name in EXPORTS:
        if name not in ("pcc_status_string", "pcc_last_error"):
            getattr(L, name).restype = ci
    _lib = L
    return L


def sweep_plan(ntau, c0, c1, shoot_both_sides=False):
    """The sweep slots (2 column + side) a pipeline over columns [c0, c1)
    marches (pcc_sweep_plan; needs no device)."""
    L = load()
    n = L.pcc_sweep_plan(int(ntau), int(bool(shoot_both_sides)), int(c0), int(c1), None, 0)
    if n < 0:
        raise PccError(PCC_ERR_INVALID_ARG, "pcc_sweep_plan: invalid Ntau or column range")
    out = np.zeros(n, dtype=np.int32)
    L.pcc_sweep_plan(int(ntau), int(bool(shoot_both_sides)), int(c0), int(c1), out.ctypes.data_as(_I), n)
    return out


def _p(a):
    return a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Engine:
    """A pcc_ctx: one CUDA device and one stream."""

    def __init__(self, device=0):
        self.lib = load()
        self.ctx = ctypes.c_void_p()
        self._solves = weakref.WeakSet()
        self._check(self.lib.pcc_ctx_create(device, None, ctypes.byref(self.ctx)), ctx=False)

    def _check(self, st, ctx=True):
        if st != 0:
            msg = self.lib.pcc_last_error(self.ctx).decode() if ctx and self.ctx else ""
            raise PccError(st, msg)

    def close(self):
        """Destroys the context; solves created from it are closed first."""
        for s in list(self._solves):
            s.close()
        if self.ctx:
            self.lib.pcc_ctx_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, desc):
        if isinstance(desc, dict):
            desc = SolveDesc.from_config(desc)
        s = Solve(self, desc)
        self._solves.add(s)
        return s

    def rhs_eval(self, ntau, dim, y, x):
        y = _f64(y).reshape(-1, ntau)
        x = _f64(np.atleast_1d(x))
        out = np.zeros_like(y)
        self._check(self.lib.pcc_rhs_eval(self.ctx, ntau, dim, y.shape[0], _p(y), _p(x), _p(out)))
        return out

    def irk_step(self, ntau, dim, scheme, precision, max_its, y, x_in, x_out):
        y = _f64(y).reshape(-1, ntau)
        xi = _f64(np.atleast_1d(x_in))
        xo = _f64(np.atleast_1d(x_out))
        out = np.zeros_like(y)
        its = np.zeros(y.shape[0], dtype=np.int32)
        self._check(self.lib.pcc_irk_step(self.ctx, ntau, dim, scheme, precision, max_its, y.shape[0], _p(y),
                                          _p(xi), _p(xo), _p(out), its.ctypes.data_as(_I)))
        return out, its

    def lu_solve(self, A, b, precision=PREC_FP64):
        A = _f64(A)
        b = _f64(b)
        x = np.zeros_like(b)
        rep = RefineReport()
        self._check(self.lib.pcc_lu_solve(self.ctx, b.size, _p(A), _p(b), _p(x), precision, ctypes.byref(rep)))
        return x, rep.as_dict()

    def pack(self, ntau, up, psic, fc):
        """packSpectralFields(U_p, psi_c, f_c) -> z (Nnewton reals)."""
        a, b, c = _f64(up), _f64(psic), _f64(fc)
        z = np.zeros(3 * ntau // 4)
        self._check(self.lib.pcc_pack_fields(self.ctx, ntau, _p(a), _p(b), _p(c), _p(z)))
        return z

    def unpack(self, ntau, z):
        """unpackSpectralFields(z) -> (U_p, psi_c, f_c)."""
        z = _f64(z)
        up, ps, fc = np.zeros(ntau), np.zeros(ntau), np.zeros(ntau)
        self._check(self.lib.pcc_unpack_fields(self.ctx, ntau, _p(z), _p(up), _p(ps), _p(fc)))
        return up, ps, fc

    def expansions(self, ntau, dim, delta, xl, xr, fc, psic, up):
        """(Y_left, Y_right) from time-domain fields."""
        a, b, c = _f64(fc), _f64(psic), _f64(up)
        yl, yr = np.zeros(ntau), np.zeros(ntau)
        self._check(self.lib.pcc_expansions(self.ctx, ntau, dim, delta, xl, xr, _p(a), _p(b), _p(c), _p(yl),
                                            _p(yr)))
        return yl, yr

    def dft(self, x, sign):
        """Unscaled DFT exp(sign 2 pi i jk/n) of complex rows of x."""
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.complex128)
        out = np.zeros_like(x)
        self._check(self.lib.pcc_dft(self.ctx, x.shape[1], x.shape[0], sign, x.ctypes.data_as(_D),
                                     out.ctypes.data_as(_D)))
        return out

    @staticmethod
    def _ptrs(items):
        return (ctypes.c_void_p * len(items))(*[ctypes.c_void_p(x) for x in items])

    def jacobian_batch(self, solves, in0s, out0s, stats=None):
        """assembleJacobian for several solves in one batch launch -> list of J."""
        ins = [_f64(a) for a in in0s]
        outs = [_f64(a) for a in out0s]
        Js = [np.zeros((a.size, a.size)) for a in ins]
        st = stats if stats is not None else Stats()
        self._check(self.lib.pcc_jacobian_batch(
            self.ctx, len(solves), self._ptrs([s.h.value for s in solves]),
            self._ptrs([a.ctypes.data for a in ins]), self._ptrs([a.ctypes.data for a in outs]),
            self._ptrs([J.ctypes.data for J in Js]), ctypes.byref(st)))
        return Js

    def newton_iterate(self, solves, precision=PREC_FP64, stats=None):
        """One device-resident Newton iteration of every running solve -> states."""
        states = (NewtonState * len(solves))()
        st = stats if stats is not None else Stats()
        self._check(self.lib.pcc_newton_iterate(self.ctx, len(solves), self._ptrs([s.h.value for s in solves]),
                                                precision, states, ctypes.byref(st)))
        return [x.as_dict() for x in states]

    def newton_solve(self, solves, in0s, precision=PREC_FP64, stats=None):
        """NewtonSolver::run for several solves at once -> (results, states)."""
        xs = [_f64(a).copy() for a in in0s]
        states = (NewtonState * len(solves))()
        st = stats if stats is not None else Stats()
        self._check(self.lib.pcc_newton_solve(self.ctx, len(solves), self._ptrs([s.h.value for s in solves]),
                                              self._ptrs([x.ctypes.data for x in xs]), precision, states,
                                              ctypes.byref(st)))
        return xs, [x.as_dict() for x in states]

    def resample(self, fields, ntau_out):
        """create_simulation_data.py double(), repeated: rows of Ntau samples -> ntau_out samples."""
        x = _f64(np.atleast_2d(fields))
        out = np.zeros((x.shape[0], ntau_out))
        self._check(self.lib.pcc_resample_fields(self.ctx, x.shape[1], ntau_out, x.shape[0], _p(x), _p(out)))
        return out

    def double_config(self, cfg):
        """create_simulation_data.py create_doub_input for one configuration:
        Ntau doubled, fields resampled, Converged false."""
        c = dict(cfg)
        ic = dict(c["Initial_Conditions"])
        n = int(c["Ntau"])
        f = self.resample(np.array([ic["fc"], ic["psic"], ic["Up"]]), 2 * n)
        ic["fc"], ic["psic"], ic["Up"] = f[0].tolist(), f[1].tolist(), f[2].tolist()
        c["Initial_Conditions"] = ic
        c["Ntau"] = 2 * n
        c["Converged"] = False
        return c

    # -- serving ---------------------------------------------------------------
    def serve_start(self, hbm_budget_bytes=0, max_active=0):
        opts = ServeOpts(int(hbm_budget_bytes), int(max_active))
        self._check(self.lib.pcc_serve_start(self.ctx, ctypes.byref(opts)))

    def submit(self, cfg, in0, precision=PREC_FP64):
        """Queues one Newton solve (a SimulationConfig dict or SolveDesc) -> ticket."""
        desc = SolveDesc.from_config(cfg) if isinstance(cfg, dict) else cfg
        x = _f64(in0)
        req = Request(desc, _p(x), int(precision))
        t = ctypes.c_uint64(0)
        self._check(self.lib.pcc_submit(self.ctx, ctypes.byref(req), ctypes.byref(t)))
        self._ticket_nn = getattr(self, "_ticket_nn", {})
        self._ticket_nn[t.value] = 3 * desc.ntau // 4
        return t.value

    def _result(self, fn, ticket, *args):
        r = Result()
        x = np.zeros(self._ticket_nn[ticket])
        st = fn(self.ctx, ctypes.c_uint64(ticket), *args, ctypes.byref(r), _p(x))
        if st != PCC_ERR_TIMEOUT:
            self._check(st)
        d = r.as_dict()
        return d, (x if r.done else None)

    def poll(self, ticket):
        """-> (result dict, x or None while running)."""
        return self._result(self.lib.pcc_poll, ticket)

    def wait(self, ticket, timeout_s=600.0):
        """As poll, blocking up to timeout_s; on timeout x is None and done is 0."""
        return self._result(self.lib.pcc_wait, ticket, ctypes.c_double(timeout_s))

    def serve_stats(self):
        info = ServeInfo()
        self._check(self.lib.pcc_serve_stats(self.ctx, ctypes.byref(info)))
        return info.as_dict()

    def serve_stop(self):
        self._check(self.lib.pcc_serve_stop(self.ctx))

    def march_tuning(self, ntau, stages=2):
        """The autotuned transform schedule: {'pair': 0/1, 'ms_pair', 'ms_single'}."""
        pair = ctypes.c_int(0)
        mp, ms = ctypes.c_double(0), ctypes.c_double(0)
        self._check(self.lib.pcc_march_tuning(self.ctx, ntau, stages, ctypes.byref(pair), ctypes.byref(mp),
                                              ctypes.byref(ms)))
        return {"pair": pair.value, "ms_pair": mp.value, "ms_single": ms.value}

    def fp64_peak_tflops(self):
        v = ctypes.c_double(0)
        self._check(self.lib.pcc_fp64_peak(self.ctx, ctypes.byref(v)))
        return v.value


class Solve:
    """A pcc_solve: device buffers, grid and tables for one SimulationConfig."""

    def __init__(self, engine, desc):
        self.engine = engine
        self.lib = engine.lib
        self.desc = desc
        self.ntau = desc.ntau
        self.nn = 3 * desc.ntau // 4
        self.h = ctypes.c_void_p()
        engine._check(self.lib.pcc_solve_create(engine.ctx, ctypes.byref(desc), ctypes.byref(self.h)))

    def close(self):
        # a closed engine has already destroyed this solve with its context
        if self.h and self.engine.ctx:
            self.lib.pcc_solve_destroy(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_grid(self, grid):
        g = _f64(grid)
        self.engine._check(self.lib.pcc_solve_set_grid(self.h, _p(g)))

    def grid(self):
        g = np.zeros(self.desc.nl + self.desc.nr + 1)
        self.engine._check(self.lib.pcc_solve_grid(self.h, _p(g)))
        return g

    def shoot(self, in0, stats=None):
        in0 = _f64(in0)
        out = np.zeros(self.nn)
        st = Stats()
        r = self.lib.pcc_shoot(self.h, _p(in0), _p(out), ctypes.byref(st))
        if stats is not None:
            stats.update(st.as_dict())  # on a failure too: fail_side / fail_grid_index locate it
        self.engine._check(r)
        return out

    def jacobian(self, in0, out0, stats=None):
        in0, out0 = _f64(in0), _f64(out0)
        J = np.zeros((self.nn, self.nn))
        st = Stats()
        r = self.lib.pcc_jacobian(self.h, _p(in0), _p(out0), _p(J), ctypes.byref(st))
        if stats is not None:
            stats.update(st.as_dict())  # on a failure too
        self.engine._check(r)
        return J

    def jacobian_columns(self, in0, out0, c0, c1, stats=None):
        """Columns [c0, c1) as an (nn, c1-c0) array (column nn = base output)."""
        in0 = _f64(in0)
        out0 = _f64(out0) if out0 is not None else None
        cols = np.zeros((c1 - c0, self.nn))
        st = Stats()
        r = self.lib.pcc_jacobian_columns(self.h, _p(in0), _p(out0) if out0 is not None else None, c0, c1,
                                          _p(cols), ctypes.byref(st))
        if stats is not None:
            stats.update(st.as_dict())  # on a failure too
        self.engine._check(r)
        return cols.T.copy()

    def jacobian_device(self, d_in0, d_out0, d_J):
        """Asynchronous build on device pointers (ints); pair with sync()."""
        self.engine._check(self.lib.pcc_jacobian_device(self.h, ctypes.c_void_p(d_in0), ctypes.c_void_p(d_out0),
                                                        ctypes.c_void_p(d_J)))

    def jacobian_columns_device(self, d_in0, d_out0, c0, c1, d_cols):
        """Columns [c0, c1) into device memory d_cols, column-major; finish with sync()."""
        self.engine._check(self.lib.pcc_jacobian_columns_device(self.h, ctypes.c_void_p(d_in0),
                                                                ctypes.c_void_p(d_out0), c0, c1,
                                                                ctypes.c_void_p(d_cols)))

    def sync(self):
        st = Stats()
        self.engine._check(self.lib.pcc_solve_sync(self.h, ctypes.byref(st)))
        return st.as_dict()

    def newton_step(self, in0, precision=PREC_FP64):
        """One NewtonSolver::run iteration; returns (new in0, err, stats, report)."""
        x = _f64(in0).copy()
        err = ctypes.c_double(0)
        st, rep = Stats(), RefineReport()
        self.engine._check(self.lib.pcc_newton_step(self.h, _p(x), ctypes.byref(err), precision, ctypes.byref(st),
                                                    ctypes.byref(rep)))
        return x, err.value, st.as_dict(), rep.as_dict()

    def shoot_debug(self, in0, debug_nx):
        """shoot + the Debug field export -> (out0, grid indices, fields[k][4][Ntau] = A, U, V, f)."""
        x = _f64(in0)
        out = np.zeros(self.nn)
        cnt = ctypes.c_int(0)
        # the first call only counts the snapshots
        self.lib.pcc_shoot_debug(self.h, _p(x), _p(out), int(debug_nx), 0, ctypes.byref(cnt), None, None, None)
        k = cnt.value
        idx = np.zeros(k, dtype=np.int32)
        fields = np.zeros((k, 4, self.ntau))
        self.engine._check(self.lib.pcc_shoot_debug(self.h, _p(x), _p(out), int(debug_nx), k, ctypes.byref(cnt),
                                                    idx.ctypes.data_as(_I), _p(fields), None))
        return out, idx, fields

    def newton_begin(self, in0):
        self.engine._check(self.lib.pcc_newton_begin(self.h, _p(_f64(in0))))

    def newton_result(self):
        x = np.zeros(3 * self.desc.ntau // 4)
        st = NewtonState()
        self.engine._check(self.lib.pcc_newton_result(self.h, _p(x), ctypes.byref(st)))
        return x, st.as_dict()

    def boundary_data(self, in0):
        in0 = _f64(in0)
        yl, yr = np.zeros(self.ntau), np.zeros(self.ntau)
        self.engine._check(self.lib.pcc_boundary_data(self.h, _p(in0), _p(yl), _p(yr)))
        return yl, yr

    def sweep(self, y_init, sides, stats=None):
        y = _f64(y_init).reshape(-1, self.ntau)
        sd = np.ascontiguousarray(sides, dtype=np.int32)
        out = np.zeros_like(y)
        st = Stats()
        r = self.lib.pcc_sweep(self.h, y.shape[0], sd.ctypes.data_as(_I), _p(y), _p(out), ctypes.byref(st))
        if stats is not None:  # filled on failure too (the failing sweep and grid index)
            stats.update(st.as_dict())
        self.engine._check(r)
        return out


def config_from_json(path_or_dict):
    """Loads a reference simulation JSON (dict returned unchanged)."""
    if isinstance(path_or_dict, dict):
        return path_or_dict
    with open(path_or_dict) as f:
        return json.load(f)
