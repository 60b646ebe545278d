import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def small_sphere():
    from scadyn_b200 import meshgen
    return meshgen.sphere(4, seed=1, eps=2.25 + 0.01j)


@pytest.fixture(scope="session")
def small_op(small_sphere):
    """Oracle operator data for a 1680-tet sphere at ka = 1."""
    from oracle import oracle as O
    k = 1.0 / small_sphere.a
    return O.setup(small_sphere, k, grid_size=1.8, nthreads=0)


@pytest.fixture(scope="session")
def dev_small(small_op):
    """The oracle's operator of the 1680-tet sphere loaded into a device
    context with the default kernel choices (GPU tests only)."""
    from tests.gpu_helpers import solver_from_oracle
    s = solver_from_oracle(small_op)
    yield s
    s.close()


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(1234)
