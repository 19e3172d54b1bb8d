import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); parity tests proper")
    config.addinivalue_line("markers", "slow: full-grid CPU reference runs")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref_model():
    from oracle import ref
    if not ref.available():
        pytest.skip("compiled reference (oracle/_ref) not present")
    return ref.Ref.get_instance()
