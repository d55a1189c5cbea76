"""numpy restatements of the reference's Python-side and host-side helpers
around the Newton-shooting path.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the cpu_baseline
leg of bench.py may import this module, as the checker; the product never does.

Pinned by tests/golden/ref_resample_128.npz (made by importing the reference
script itself, tests/golden/make_resample_golden.py) and by
tests/golden/ref_suite_128.npz (the reference's own multiple-run mode).
"""
import numpy as np


def double_field(data):
    """scripts/create_simulation_data.py:37-58 (double): Ntau samples of a
    periodic field -> 2 Ntau samples by zero-padding the spectrum.  Kept as the
    script does it: modes 0 .. Ntau/2-2 are copied, mode Ntau/2-1 is left out
    (its partner -(Ntau/2-1) is kept, so the real part carries half of it), the
    old Nyquist mode is split in halves at +-Ntau/2, and the result is
    2 * Re ifft."""
    f = np.fft.fft(np.asarray(data, dtype=np.float64))
    nt = 2 * f.size
    d = np.zeros(nt, dtype=np.complex128)
    d[: nt // 4 - 1] = f[: nt // 4 - 1]
    d[nt // 4] = f[nt // 4] / 2
    d[3 * nt // 4] = f[nt // 4] / 2
    d[3 * nt // 4 + 1:] = f[nt // 4 + 1:]
    return np.real(np.sqrt(4) * np.fft.ifft(d))


def resample_field(data, ntau_out):
    """Repeated doubling up to ntau_out (a power-of-two multiple)."""
    x = np.asarray(data, dtype=np.float64)
    while x.size < ntau_out:
        x = double_field(x)
    if x.size != ntau_out:
        raise ValueError("ntau_out must be Ntau times a power of two")
    return x


def quadratic_extrapolate(dims, values, d):
    """src/main.cpp:300-354 with src/common.cpp:151-198: per sample, the
    quadratic a D^2 + b D + c through the last three converged runs (a 3x3
    least-squares solve, exact for distinct D) evaluated at D = d."""
    A = np.array([[x * x, x, 1.0] for x in dims])
    coef = np.linalg.lstsq(A, np.asarray(values, dtype=np.float64), rcond=None)[0]
    return coef[0] * d * d + coef[1] * d + coef[2]
