"""Test configuration.

Markers: ``gpu`` tests need a CUDA device (a B200); everything else runs on
the CPU.  The oracle (test infrastructure) is built on demand.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size (2^28) property checks")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def golden_cases():
    import numpy as np

    data = np.load(GOLDEN / "chase_cases.npz")
    names = sorted({k.split("__")[0] for k in data.files})
    out = {}
    for nm in names:
        out[nm] = {k.split("__")[1]: data[k] for k in data.files if k.startswith(nm + "__")}
    return out


@pytest.fixture(scope="session")
def kat():
    import json

    return json.loads((GOLDEN / "kat.json").read_text())
