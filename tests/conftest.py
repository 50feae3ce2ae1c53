import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def reference_dir():
    """The reference source tree, from the GALE_REFERENCE_DIR environment variable; the
    tests that read the reference's own files skip when it is unset or absent."""
    d = os.environ.get("GALE_REFERENCE_DIR")
    if not d or not os.path.isdir(d):
        pytest.skip("GALE_REFERENCE_DIR is not set to the reference source tree")
    return d


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
