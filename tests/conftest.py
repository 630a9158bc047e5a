"""Shared test set-up: import paths, the ``gpu`` marker and fixture loaders."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "lfm-physics_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running parity run")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def golden_json(arr) -> dict:
    return json.loads(str(arr))


@pytest.fixture(scope="session")
def cuda_device():
    """The first CUDA device; GPU tests fail loudly when it is absent."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("test marked gpu needs a CUDA device")
    return torch.device("cuda:0")
