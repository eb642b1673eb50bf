"""Shared pytest setup: the `gpu` marker, import paths, golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and libcasphy.so")


@pytest.fixture(scope="session")
def golden():
    """(cases, reference_outputs) from tests/golden/."""
    d = os.path.join(ROOT, "tests", "golden")
    z = np.load(os.path.join(d, "cases.npz"))
    cases = {}
    for k in z.files:
        kind, name, field = k.split("/")
        cases.setdefault((kind, name), {})[field] = z[k]
    ref = dict(np.load(os.path.join(d, "reference_outputs.npz")))
    return cases, ref


@pytest.fixture(scope="session")
def gpu_lib():
    """libcasphy loaded on a visible GPU (tests marked gpu only)."""
    import casphy_b200.lib as L
    L.lib()
    return L


@pytest.fixture(params=["1", "8"])
def stale_batch(request, monkeypatch):
    """Run a join test with one stale rescan per phase (the sequential
    schedule, whose counts equal the oracle's) and with batches of up to 8."""
    monkeypatch.setenv("CASPHY_STALE_BATCH", request.param)
    return int(request.param)
