import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def cflib():
    from cudafusion_b200 import build

    build.build()
    from cudafusion_b200 import _lib

    return _lib.lib()


def reference_dir():
    """The CUDAFusion checkout, where one is on this machine: CF_REFERENCE_DIR,
    else a `reference` directory beside this repository.  None when absent
    (tests that compile or run the reference's sources then skip)."""
    d = os.environ.get("CF_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")
    return d if os.path.isdir(os.path.join(d, "include")) else None
