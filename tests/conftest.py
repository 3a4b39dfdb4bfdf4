import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "ternary-chns_b200"), os.path.join(ROOT, "tests"),
          os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a) and the built extension")
    config.addinivalue_line("markers", "slow: long CPU run, enabled with CHNS_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("CHNS_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow; set CHNS_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)
