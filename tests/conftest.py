import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA engine)")


def _has_gpu():
    try:
        import harvest_cuda_b200 as hv
        return hv.cuda_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Skips GPU-marked tests cleanly when no supported GPU is visible."""
    if not _has_gpu():
        pytest.skip("no supported GPU visible")
    return True


@pytest.fixture(scope="session")
def checker():
    """The CPU checker: the reference's own WORLD build when present, else
    the C restatement."""
    import oracle
    return oracle.best()
