"""Test configuration: import paths and the ``gpu`` marker.

Tests marked ``gpu`` need a CUDA device and the built library; everything
else runs on the CPU.  ``oracle/`` is imported only here, as the checker.
"""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "fly-in-silico_b200", ROOT / "tests", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libfis_b200.so")


def cuda_ok():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def get(name):
        return np.load(ROOT / "tests" / "golden" / ("%s.npz" % name))

    return get
