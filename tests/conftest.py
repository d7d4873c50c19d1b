import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"
GOLDEN_NAMES = ["g4d", "g4d_iso", "g3d", "g2d"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the sm_100a library")


def load_golden(name: str) -> dict:
    d = np.load(GOLDEN / f"{name}.npz")
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def ctx():
    from latticeu1_b200 import Context
    return Context(0)


@pytest.fixture(params=GOLDEN_NAMES)
def golden(request):
    return request.param, load_golden(request.param)
