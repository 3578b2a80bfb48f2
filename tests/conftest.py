import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


# The reference's test scenario (tests/test_particle_filter.py:24-48 of the
# reference project), extracted by tests/golden/make_golden.py.
_FIX = json.loads((Path(__file__).resolve().parent / "golden" / "tokyo_fixture.json").read_text())
TOKYO_TRUE_POS = np.array(_FIX["true_pos"])
TOKYO_TRUE_CB = float(_FIX["true_cb"])
TOKYO_SATS = np.array(_FIX["sat_ecef"])
TOKYO_PR = np.array(_FIX["pseudoranges"])
N_TEST = int(_FIX["n_test"])
SEED = int(_FIX["seed"])


def tokyo_scenario():
    return TOKYO_SATS.copy(), TOKYO_PR.copy(), np.ones(len(TOKYO_SATS)), TOKYO_TRUE_POS.copy(), TOKYO_TRUE_CB


@pytest.fixture
def tokyo():
    return tokyo_scenario()
