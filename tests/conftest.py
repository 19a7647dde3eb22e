import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib_built():
    """The in-tree CUDA library (built here when missing; never a fallback)."""
    from anacapa_b200 import build
    build.build()
    from anacapa_b200 import api
    return api.lib()


@pytest.fixture(scope="session")
def restate_built():
    """This repository's CPU restatement of the path (oracle/restate), built here."""
    from oracle import restatebind as P
    P.build()
    return P


@pytest.fixture(scope="session")
def ref_built():
    """The reference hot path compiled from its own sources (oracle/_ref)."""
    from oracle import refbind as R
    if not (R.available("record") and R.available("nocontract")):
        if not R.build():
            pytest.skip("reference oracle not built and the reference tree is absent")
    return R


@pytest.fixture(scope="session")
def gpu(lib_built):
    if not _cuda_available():
        pytest.skip("no CUDA device")
    return lib_built
