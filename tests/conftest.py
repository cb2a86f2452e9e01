"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
CPU (oracle vs golden vectors, planner host logic, C-ABI exports)."""
from __future__ import annotations

import ctypes
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

VARIANTS = [(tr, ul) for tr in (0, 1) for ul in (0, 1)]  # transr 0=N, uplo 0=L


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(ROOT / "tests" / "golden" / "lapack_rfp.npz"))


@pytest.fixture(scope="session")
def orc():
    import oracle.oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def hostsim():
    subprocess.run(["make", "-s", "-C", str(ROOT / "tests" / "hostsim")], check=True)
    return ctypes.CDLL(str(ROOT / "tests" / "hostsim" / "libhostsim.so"))


@pytest.fixture(scope="session")
def curfp():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    import curfp_b200
    curfp_b200._lib.load()
    return curfp_b200
