"""Serving: whole Newton solves submitted over time (pcc_submit / pcc_poll /
pcc_wait), admitted by device-memory footprint, their sweeps batched into
shared launches as they become ready.

The property that matters for continuous batching: a request's result is the
same alone and in a mix with requests of other sizes that arrive while it
runs (bit for bit here, since every sweep and every per-solve kernel does the
same arithmetic wherever it runs)."""
import time

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu


def _cfg(d, **over):
    c = dict(d["cfg"])
    c.update(over)
    return c


def _islot(x):
    return 2 * x.size // 3 + 2


def test_serve_same_alone_and_in_mix(engine):
    c1, c2 = load_case("c1_newton"), load_case("c2_fixture")
    cfg1 = _cfg(c1, PrecisionNewton=1e-12, MaxIterNewton=12)
    engine.serve_start()
    try:
        t = engine.submit(cfg1, c1["in0"])
        alone, x_alone = engine.wait(t)
        assert alone["done"] == 1 and alone["status"] == 0, alone
        assert alone["newton"]["state"] == "CONVERGED"
        ref = c1["x_star"]
        i = _islot(ref)
        assert abs(x_alone[i] / ref[i] - 1) < 1e-10

        # the mix: a larger solve first, then the same request twice, staggered
        t_big = engine.submit(_cfg(c2, PrecisionNewton=1e-30, MaxIterNewton=2), c2["in0"])
        time.sleep(0.05)
        t_a = engine.submit(cfg1, c1["in0"])
        time.sleep(0.02)
        t_b = engine.submit(cfg1, c1["in0"])
        ra, xa = engine.wait(t_a)
        rb, xb = engine.wait(t_b)
        rbig, _ = engine.wait(t_big)
        assert np.array_equal(xa, x_alone) and np.array_equal(xb, x_alone)
        assert ra["newton"]["iterations"] == alone["newton"]["iterations"]
        assert ra["newton"]["err"] == alone["newton"]["err"]
        assert rbig["newton"]["state"] == "MAX_ITER" and rbig["newton"]["iterations"] == 2
        assert rbig["status"] == 10  # PCC_ERR_NEWTON_NO_CONVERGENCE, as the reference's exit
        st = engine.serve_stats()
        assert st["completed"] == 4 and st["launches"] >= 1 and st["sweeps"] > 0
    finally:
        engine.serve_stop()


def test_serve_admission_by_memory_budget(engine):
    c1 = load_case("c1_fixture")
    cfg = _cfg(c1, PrecisionNewton=1e-30, MaxIterNewton=2)
    engine.serve_start()
    t = engine.submit(cfg, c1["in0"])
    r0, x0 = engine.wait(t)
    fp = r0["footprint_bytes"]
    engine.serve_stop()
    assert fp > 0
    # room for one such solve at a time: the others wait for its memory
    engine.serve_start(hbm_budget_bytes=int(fp * 1.5))
    try:
        ts = [engine.submit(cfg, c1["in0"]) for _ in range(3)]
        peak = 0
        while True:
            st = engine.serve_stats()
            peak = max(peak, st["bytes_in_use"])
            if st["completed"] == 3:
                break
            time.sleep(0.005)
        res = [engine.wait(t) for t in ts]
        assert peak <= int(fp * 1.5)
        for r, x in res:
            assert r["done"] == 1 and np.array_equal(x, x0)
        q = sorted(r["ms_queued"] for r, _ in res)
        assert q[2] > q[0]  # the last one waited for memory
    finally:
        engine.serve_stop()


def test_serve_rejects_solve_larger_than_budget(engine):
    c1 = load_case("c1_fixture")
    engine.serve_start(hbm_budget_bytes=1 << 20)
    try:
        r, x = engine.wait(engine.submit(_cfg(c1), c1["in0"]))
        assert r["done"] == 1 and r["status"] == 3  # PCC_ERR_OOM
    finally:
        engine.serve_stop()


def test_serve_reports_irk_failure(engine):
    c1 = load_case("c1_fixture")
    engine.serve_start()
    try:
        r, x = engine.wait(engine.submit(_cfg(c1, MaxIterIRK=1), c1["in0"]))
        assert r["done"] == 1 and r["status"] == 4 and r["newton"]["state"] == "IRK_FAILED"
        assert np.array_equal(x, c1["in0"])
    finally:
        engine.serve_stop()


def test_serve_wait_times_out_and_rejects_non_finite_input(engine):
    """pcc_wait returns PCC_ERR_TIMEOUT (result not done) when the solve has
    not ended by its deadline, and the solve still completes; a request whose
    free data hold a NaN is refused at submission with PCC_ERR_NAN."""
    import ctypes

    import pcc

    c1 = load_case("c1_newton")
    engine.serve_start()
    try:
        t = engine.submit(_cfg(c1, PrecisionNewton=1e-12, MaxIterNewton=12), c1["in0"])
        r = pcc.Result()
        x = np.zeros(c1["in0"].size)
        st = engine.lib.pcc_wait(engine.ctx, ctypes.c_uint64(t), ctypes.c_double(0.0), ctypes.byref(r),
                                 x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert st == pcc.PCC_ERR_TIMEOUT and r.done == 0
        res, xs = engine.wait(t)
        assert res["done"] == 1 and res["status"] == 0 and xs is not None
        bad = c1["in0"].copy()
        bad[5] = np.nan
        with pytest.raises(pcc.PccError) as e:
            engine.submit(_cfg(c1), bad)
        assert e.value.status == pcc.PCC_ERR_NAN
    finally:
        engine.serve_stop()


def test_serve_stop_while_waiting_and_results_delivered_once(engine):
    """pcc_serve_stop overlapping a pcc_wait and a pcc_poll loop on other
    threads: the waiter still receives its result (stop finishes every
    submitted request first), the poller ends with PCC_ERR_INVALID_ARG once the
    server is gone, and nothing blocks.  A delivered result is released: the
    ticket is unknown afterwards."""
    import ctypes
    import threading

    import pcc

    c1 = load_case("c1_newton")
    cfg = _cfg(c1, PrecisionNewton=1e-12, MaxIterNewton=12)
    engine.serve_start()
    t_done = engine.submit(cfg, c1["in0"])
    r, _ = engine.wait(t_done)
    assert r["done"] == 1
    with pytest.raises(pcc.PccError) as e:
        engine.poll(t_done)  # delivered once
    assert e.value.status == pcc.PCC_ERR_INVALID_ARG

    t = engine.submit(cfg, c1["in0"])
    got, polled = {}, {}

    def waiter():
        got["r"], got["x"] = engine.wait(t, 600.0)

    def poller():
        res = pcc.Result()
        codes = set()
        while not got.get("stopped"):
            codes.add(engine.lib.pcc_poll(engine.ctx, ctypes.c_uint64(t + 1000), ctypes.byref(res), None))
            time.sleep(0.001)
        codes.add(engine.lib.pcc_poll(engine.ctx, ctypes.c_uint64(t + 1000), ctypes.byref(res), None))
        polled["codes"] = codes

    th_w, th_p = threading.Thread(target=waiter), threading.Thread(target=poller)
    th_w.start()
    th_p.start()
    time.sleep(0.05)
    engine.serve_stop()
    got["stopped"] = True
    th_w.join(60)
    th_p.join(60)
    assert not th_w.is_alive() and not th_p.is_alive()
    assert got["r"]["done"] == 1 and got["r"]["status"] == 0 and got["x"] is not None
    assert polled["codes"] <= {pcc.PCC_ERR_INVALID_ARG}  # unknown ticket before and after the stop


def test_first_submits_from_two_threads_start_one_loop():
    """Serving starts lazily inside the first pcc_submit; two threads that
    submit at the same moment on a fresh context both get their requests
    queued (no PCC_ERR_BUSY from a second start) and both results arrive."""
    import threading

    import pcc

    c1 = load_case("c1_newton")
    cfg = _cfg(c1, PrecisionNewton=1e-12, MaxIterNewton=12)
    eng = pcc.Engine(0)
    try:
        go = threading.Barrier(2)
        tickets, errors = [], []

        def submit():
            go.wait()
            try:
                tickets.append(eng.submit(cfg, c1["in0"]))
            except pcc.PccError as e:
                errors.append(e)

        ths = [threading.Thread(target=submit) for _ in range(2)]
        for th in ths:
            th.start()
        for th in ths:
            th.join(60)
        assert not errors and len(tickets) == 2 and tickets[0] != tickets[1]
        xs = []
        for t in tickets:
            r, x = eng.wait(t, 600.0)
            assert r["done"] == 1 and r["status"] == 0
            xs.append(x)
        assert np.array_equal(xs[0], xs[1])
        eng.serve_stop()
    finally:
        eng.close()
