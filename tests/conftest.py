import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def ref_lib():
    """The reference's own sources compiled on the host (oracle/_ref); skipped
    where it was not built."""
    from oracle.refbuild import build_ref
    try:
        return build_ref.load()
    except FileNotFoundError as e:
        pytest.skip(str(e))
