"""Shared fixtures.  Tests marked `gpu` need a CUDA device (B200); the rest
run on the CPU: the oracle against its pins and golden fixtures, the host
logic, and the C ABI surface of the library."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


def rel_l2(a, b) -> float:
    import numpy as np
    a = [np.asarray(x) for x in (a if isinstance(a, (list, tuple)) else [a])]
    b = [np.asarray(x) for x in (b if isinstance(b, (list, tuple)) else [b])]
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return (num / den) ** 0.5 if den > 0 else num ** 0.5
