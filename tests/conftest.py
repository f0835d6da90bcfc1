import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C ABI")


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle
    p = oracle.reference_path()
    if p is None:
        pytest.skip("reference library not built on this host (oracle/_ref)")
    return oracle.Reference(p)


@pytest.fixture(scope="session")
def ms():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import engine_b200
    return engine_b200


@pytest.fixture(scope="session")
def arena(ms):
    a = ms.Arena(int(os.environ.get("MS_TEST_ARENA", str(24 << 30))))
    yield a
    a.close()
