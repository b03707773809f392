import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


@pytest.fixture(scope="session")
def oracle_mod():
    """The CPU oracle package, with its restatement built (and the reference
    build when the reference tree is present)."""
    import oracle
    oracle.build(reference=True)
    return oracle


@pytest.fixture(scope="session")
def bm3d_lib():
    """The product library (built in-tree)."""
    from isp_mw_b200 import build as b
    b.build()
    import isp_mw_b200
    return isp_mw_b200.load_library()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
