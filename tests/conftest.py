import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libdpd_b200.so")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"ref_{name}.npz")))


def force_err(f, f_ref):
    """Largest per-particle force error relative to the RMS particle force."""
    d = np.linalg.norm(np.asarray(f) - np.asarray(f_ref), axis=1)
    rms = np.sqrt((np.linalg.norm(f_ref, axis=1) ** 2).mean())
    return d.max() / rms


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.load()
    return oracle
