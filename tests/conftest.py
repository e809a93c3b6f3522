import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a B200)")

import pytest

PKG = os.path.join(os.path.dirname(HERE), "bullet-physics_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)


@pytest.fixture(scope="session")
def bgpu_mod():
    import bgpu

    bgpu.lib()
    return bgpu


@pytest.fixture(scope="session")
def gpu(bgpu_mod):
    if bgpu_mod.device_count() == 0:
        pytest.fail("GPU test collected on a machine without a CUDA device (run with -m 'not gpu')")
    return bgpu_mod
