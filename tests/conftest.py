import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
SCENE_NAMES = ("mixed", "air_pml", "fields")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    with np.load(GOLDEN / f"golden_{name}.npz", allow_pickle=False) as data:
        return {k: data[k] for k in data.files}


@pytest.fixture(params=SCENE_NAMES)
def golden(request):
    g = load_golden(request.param)
    g["name"] = request.param
    return g
