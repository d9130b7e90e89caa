import functools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libluna_b200.so")


@functools.lru_cache(maxsize=None)
def jittered_mesh(nx: int, dim: int = 3, jitter: float = 0.1, seed: int = 1):
    from luna_cpp_b200.mesh import build_mesh, jittered_points

    cells = (nx,) * dim
    return build_mesh(jittered_points(cells, jitter=jitter, seed=seed), box=(1.0,) * dim)


@functools.lru_cache(maxsize=None)
def random_mesh(n: int, dim: int = 3, seed: int = 5):
    from luna_cpp_b200.mesh import build_mesh

    pts = np.random.default_rng(seed).random((n, dim))
    return build_mesh(pts, box=(1.0,) * dim)


@pytest.fixture(scope="session")
def mesh16():
    return jittered_mesh(16)


@pytest.fixture(scope="session")
def mesh32():
    return jittered_mesh(32)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=False)
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from luna_cpp_b200 import hydro

    hydro.lib()
    return True
