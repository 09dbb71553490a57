import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C-ABI")
    config.addinivalue_line("markers", "slow: longer CPU-side oracle checks")


@pytest.fixture(scope="session")
def pins():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "reference_pins.json")) as f:
        return json.load(f)
