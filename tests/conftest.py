import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(autouse=True)
def libm_math_by_default():
    """The oracle's arc cosine is process-wide: libm (as the reference) unless a
    test asks for the library's portable one (GPU check mode)."""
    from oracle.bridge import PortCloth, available
    if available("port"):
        PortCloth.set_portable_math(False)
    yield
    if available("port"):
        PortCloth.set_portable_math(False)


@pytest.fixture(scope="session")
def ref_threads():
    from oracle.bridge import RefCloth, available
    if available("ref"):
        RefCloth.set_threads(1)
    return 1
