import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)  # tests/golden/inputs.py is imported as golden.inputs


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 host)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build(reference=True)
    return oracle.Oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle
    if not oracle.Reference.available():
        pytest.skip("reference CPU codec (oracle/_ref) was not built here")
    return oracle.Reference()


@pytest.fixture(scope="session")
def cuda_ready():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    torch.cuda.init()
    return torch
