"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "reference: needs oracle/_ref (the reference compiled from its sources)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def golden():
    data = np.load(GOLDEN / "reference_fixtures.npz")
    meta = json.loads((GOLDEN / "reference_fixtures.json").read_text())
    return data, meta


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.oracle_lib()
    return O


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine library; GPU tests only."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    import cfd_solvers_b200 as cs

    return cs
