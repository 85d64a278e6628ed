import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_ls.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def built_library():
    """Path of liblippmannschwinger.so, building it (and libfibres.so) if either is missing."""
    from jaxmaterials_b200 import _lib

    path = _lib.library_path()
    fibres = os.path.join(os.path.dirname(path), _lib.FIBRES_NAME)
    if not os.path.exists(path) or not os.path.exists(fibres):
        subprocess.run(["make", "-C", os.path.join(ROOT, "jaxmaterials_b200", "csrc")],
                       check=True, capture_output=True)
    return path


def reference_material(shape, seed=784173):
    """(lmbda, mu) as bound by the reference test (tests/test_lippmann_schwinger.py:37-47,
    75): initialise_material returns (first draw, second draw)."""
    rng = np.random.default_rng(seed=seed)
    first = np.ones(shape) + rng.uniform(size=shape, low=-0.2, high=0.2)
    second = np.ones(shape) + rng.uniform(size=shape, low=-0.2, high=0.2)
    return first, second
