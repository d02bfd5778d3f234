import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_ref():
    """The reference's own CPU code (oracle/_ref), or skip when not built."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return ref
