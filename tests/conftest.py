import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libne_cuda.so path")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def oracle_cls():
    """The strongest oracle available: the reference compiled in place, else
    the C restatement (both are pinned to each other by the CPU suite)."""
    from oracle import oracle as O
    if O.ref_available():
        return O.RefOracle
    if O.port_available():
        return O.PortOracle
    pytest.skip("no oracle library built (run __graft_entry__.build())")
