import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")


@pytest.fixture(scope="session")
def port():
    """The CPU restatement (built on first use)."""
    from oracle import build_oracle
    from oracle import oracle as O
    build_oracle.build_port()
    return O


@pytest.fixture(scope="session")
def ref(port):
    """The reference's own k-d tree, when its harness is available."""
    from oracle import oracle as O
    if not O.ref_available():
        from oracle import build_oracle
        build_oracle.build_ref()
    if not O.ref_available():
        pytest.skip("reference harness (oracle/_ref) not available")
    return O


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pptk_b200
    from pptk_b200 import _native
    _native.lib()  # fails loudly when the library is missing
    return pptk_b200
