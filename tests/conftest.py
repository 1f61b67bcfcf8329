import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libpremixfem_b200.so")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def native():
    from premixfem_b200 import _native
    lib = _native.load()
    if lib.pmf_device_count() < 1:
        pytest.fail("no CUDA device visible to libpremixfem_b200.so")
    return lib
