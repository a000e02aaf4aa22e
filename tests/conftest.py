import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "gecco-public_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """make sure oracle and engine libraries exist (they are built in-tree)"""
    import binding
    import gccu
    if not os.path.exists(binding._LIB_PATH):
        binding.build()
    if not os.path.exists(gccu.LIB_PATH):
        gccu.build()
    return True
