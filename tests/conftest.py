import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "anqi-implementation_b200"))
sys.path.insert(0, str(REPO / "tests"))
GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", params=[8, 32])
def sample(request):
    import numpy as np

    return dict(np.load(GOLDEN / f"sample_d{request.param}.npz"))
