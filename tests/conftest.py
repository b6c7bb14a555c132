"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """Build the CPU oracle restatement if its library is missing (g++ is on every box)."""
    from oracle import oracle as O
    if not os.path.exists(O.ORACLE_SO):
        import subprocess
        subprocess.check_call([os.path.join(ROOT, "oracle", "build_oracle.sh")])
    yield


def relerr(a, b):
    a = np.asarray(a); b = np.asarray(b)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "refcl_small.npz")))


@pytest.fixture(scope="session")
def sphere2():
    from baemm_b200 import meshes
    return meshes.icosphere(2)


@pytest.fixture(scope="session")
def sphere3():
    from baemm_b200 import meshes
    return meshes.icosphere(3)
