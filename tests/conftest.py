import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    """The CPU FP64 oracle (built in place on first use)."""
    from oracle import pyoracle

    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def engine():
    """The B200 engine; on a GPU box the CUDA library must load and run."""
    from fpe_option_b200 import build

    build.build_library()
    import fpe_option_b200 as fpe

    assert fpe.is_available(), "CUDA engine not usable on this GPU box"
    return fpe
