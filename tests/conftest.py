"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the built
libpcc_b200.so; everything else runs on the CPU (oracle, host logic, ABI
surface)."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
PKG = REPO / "parallel-critical-collapse_b200"
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(REPO / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def load_case(name):
    """A reference fixture (see tests/golden/make_golden.py) as a dict."""
    d = dict(np.load(GOLDEN / f"ref_{name}.npz"))
    cfg = json.loads(str(d.pop("config")))
    d["cfg"] = cfg
    return d


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib

    oracle_lib.build()
    return oracle_lib.Oracle()


@pytest.fixture(scope="session")
def engine():
    import pcc

    eng = pcc.Engine(0)
    yield eng
    eng.close()


def rel_err(a, b):
    """max |a - b| / max |b|"""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))
