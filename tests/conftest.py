import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "phys-rs_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libphysgpu.so")


@pytest.fixture(scope="session")
def ctx():
    import physgpu
    c = physgpu.Context(0)
    yield c
    c.close()
