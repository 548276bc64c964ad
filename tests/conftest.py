import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU oracle run, enabled with DMPC_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("DMPC_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle pin; set DMPC_SLOW=1")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)
