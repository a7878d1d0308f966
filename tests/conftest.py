import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def lib():
    """The CUDA library, built in-tree if needed (no fallback)."""
    from stardust_b200 import _lib, build

    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda(lib):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch


def random_particles(n, seed, empty_every=0, clustered=False):
    rng = np.random.default_rng(seed)
    if clustered:
        c = rng.random((8, 3))
        xyz = (c[rng.integers(0, 8, n)] + rng.normal(scale=0.03, size=(n, 3))) % 1.0
    else:
        xyz = rng.random((n, 3))
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = xyz
    pos[:, :3][pos[:, :3] >= 1.0] = 0.0
    pos[:, 3] = rng.random(n).astype(np.float32)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(scale=0.3, size=(n, 3))
    vel[:, 3] = np.arange(n, dtype=np.float32)  # an id carried through sort and step
    if empty_every:
        pos[::empty_every] = (-1.0, -1.0, -1.0, 0.0)
        vel[::empty_every] = 0.0
    return pos, vel
