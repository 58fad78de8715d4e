"""Shared fixtures for the test suite.

Markers: ``gpu`` tests need a CUDA device and run the sm_100a library; everything
else runs on the CPU (oracle pins, C-ABI surface, host logic, gloo multi-process).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libgbs_b200.so")


def _ensure_oracle():
    lib = ROOT / "oracle" / "liboracle.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "liboracle.so"], check=True,
                       capture_output=True)


def _ensure_library():
    lib = ROOT / "gbskernels_b200" / "libgbs_b200.so"
    if not lib.exists():
        from gbskernels_b200 import build
        build.build()


@pytest.fixture(scope="session")
def orc():
    _ensure_oracle()
    import oracle
    return oracle


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def lib():
    _ensure_library()
    from gbskernels_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def G(lib):
    import gbskernels_b200
    return gbskernels_b200


@pytest.fixture(scope="session")
def gpu(G):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return G


def golden_cases(golden, func):
    dims = golden[f"{func}_dims"]
    mats = golden[f"{func}_mats"]
    out = []
    for i, d in enumerate(dims):
        m = np.ascontiguousarray(mats[i, :d, :d])
        mp = golden[f"{func}_mp"][i]
        truth = complex(mp[0] + mp[1], mp[2] + mp[3])
        out.append((m, truth, mp, i))
    return out


def rel_err(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)
