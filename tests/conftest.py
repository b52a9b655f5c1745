import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from hero_testlib import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def emu():
    from hero_testlib import Emu
    return Emu()


@pytest.fixture(scope="session")
def gpu_lib():
    from hero_b200 import build
    build.build_library()
    from hero_b200 import load_library
    return load_library()
