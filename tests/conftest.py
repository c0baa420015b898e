"""Test configuration: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs on any host: the oracle against the reference's golden
vectors, the host logic and the C-ABI exports.  ``-m gpu`` runs the CUDA path
through libzb on a B200 and compares it with the oracle.
"""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "zoomy-jax_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def goldens():
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "reference_goldens.npz")
