"""pcc_expansions_static: the boundary expansions with no device allocation.

It serves callers that may not allocate device memory while running (a
service that reserves its whole device-memory pool at start-up, or a library
that must avoid the device synchronisation cudaFree can cause): inputs and
outputs are the caller's device buffers, and the work arrays live in a static
device array inside the library.  This test plays the caller: it allocates the
input and output buffers itself, calls the entry point twice in a row through
the C ABI, and checks each result against pcc_expansions, the allocating
entry point, to the tolerance the expansion parity tests use (1e-12
relative).  The file is collected last, so a run that stops at its first
failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu


def _interp_field(f, n):
    """Spectral (zero-padding) interpolation of a periodic real field to n samples."""
    c = np.fft.rfft(f)
    c2 = np.zeros(n // 2 + 1, dtype=complex)
    c2[: c.size - 1] = c[:-1]
    return np.fft.irfft(c2, n) * (n / f.size)


def _cases():
    """The C1 and C3 fixtures, and the C1 fields interpolated to Ntau 2048: the
    largest size the static work area holds, which fills it exactly."""
    for name in ["c1_fixture", "c3_fixture"]:
        d = load_case(name)
        n = d["cfg"]["Ntau"]
        yield name, d["cfg"], float(d["in0"][2 * (3 * n // 4) // 3 + 2]), d["unpack_fc"], d["unpack_psic"], \
            d["unpack_up"]
    d = load_case("c1_fixture")
    fc, psic, up = (_interp_field(d[k], 2048) for k in ("unpack_fc", "unpack_psic", "unpack_up"))
    yield "c1_at_2048", dict(d["cfg"], Ntau=2048), float(d["in0"][2 * d["in0"].size // 3 + 2]), fc, psic, up


def test_static_expansions_match_allocating_entry_point(engine):
    import torch

    import pcc

    lib = pcc.load()
    dev = torch.device("cuda", 0)
    for name, cfg, delta, fc, psic, up in _cases():
        n = cfg["Ntau"]
        yl_ref, yr_ref = engine.expansions(n, cfg["Dim"], delta, cfg["XLeft"], cfg["XRight"], fc, psic, up)
        t_fc, t_ps, t_up = (torch.tensor(a, dtype=torch.float64, device=dev) for a in (fc, psic, up))
        for call in range(2):
            t_yl = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
            t_yr = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            st = lib.pcc_expansions_static(engine.ctx, n, cfg["Dim"], delta, cfg["XLeft"], cfg["XRight"],
                                           ctypes.c_void_p(t_fc.data_ptr()), ctypes.c_void_p(t_ps.data_ptr()),
                                           ctypes.c_void_p(t_up.data_ptr()), ctypes.c_void_p(t_yl.data_ptr()),
                                           ctypes.c_void_p(t_yr.data_ptr()))
            assert st == 0, lib.pcc_last_error(engine.ctx)
            torch.cuda.synchronize()  # the call is asynchronous on the context stream
            yl, yr = t_yl.cpu().numpy(), t_yr.cpu().numpy()
            assert np.max(np.abs(yl - yl_ref)) / np.max(np.abs(yl_ref)) < 1e-12, (name, call)
            assert np.max(np.abs(yr - yr_ref)) / np.max(np.abs(yr_ref)) < 1e-12, (name, call)
    assert torch.cuda.current_device() == 0  # the caller's current device is left as it was


def test_static_expansions_rejects_oversize(engine):
    """Ntau above the static work area is refused before anything runs."""
    import pcc

    lib = pcc.load()
    null = ctypes.c_void_p(0)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.pcc_expansions_static(engine.ctx, 4096, 4.0, 3.4, 0.001, 0.999, dummy, dummy, dummy, dummy, null)
    assert st == 1
    assert b"2048" in lib.pcc_last_error(engine.ctx)
