"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
a CPU-only host.  The CPU checkers (oracle/) are built on demand."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long-running case")


def _ensure_oracle():
    so = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from oracle.ffi import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.ffi import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref not built (the reference sources are not in this checkout)")
    return Reference()


@pytest.fixture(scope="session")
def pic():
    """The CUDA library, initialised on device 0 (GPU tests only)."""
    import piculator_b200 as P
    P.init(0)
    return P


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU test run without a GPU"
    return torch
