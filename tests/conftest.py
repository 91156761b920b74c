import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.pyoracle import Oracle

    return Oracle("port")


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle.pyoracle import Oracle, lib_path

    if not os.path.exists(lib_path("reference")):
        pytest.skip("oracle/_ref not built (reference sources absent)")
    return Oracle("reference")
