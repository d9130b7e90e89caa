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


def wave_state_3d(mesh, seed: int = 3, noise: float = 0.01, gamma: float = 5.0 / 3.0):
    """The reference's 3D moving-step derivative state (hydro_derivatives_test.cpp:1513-1516), extensive: waves in every
    primitive at the cell centroids plus uniform noise of +- noise."""
    rng = np.random.default_rng(seed)
    c = mesh.positions + mesh.centroid
    n, k = len(c), 2 * np.pi

    def jitter():
        return noise * rng.uniform(-1, 1, n)

    rho = 1 + 0.2 * np.sin(k * c[:, 0]) + jitter()
    vx = 0.3 * np.sin(k * c[:, 1]) + jitter()
    vy = 0.2 * np.cos(k * c[:, 2]) + jitter()
    vz = 0.25 * np.sin(k * (c[:, 0] + c[:, 2])) + jitter()
    P = 1 + 0.2 * np.cos(k * (c[:, 0] + c[:, 1] + c[:, 2])) + jitter()
    U = np.stack([rho, rho * vx, rho * vy, rho * vz, P / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)], -1)
    return U * mesh.volume[:, None]


def wave_state_2d(mesh, seed: int = 3, noise: float = 0.01, gamma: float = 5.0 / 3.0):
    """The reference's moving-step derivative state (hydro_derivatives_test.cpp:1505-1516), extensive: smooth waves in
    every primitive at the cell centroids plus uniform noise of +- noise in each, so no two neighbours tie and no field is
    uniform (a uniform field leaves the limiter's pattern and its scale (bound - W_i) / (g0 . o) to rounding)."""
    rng = np.random.default_rng(seed)
    c = mesh.positions + mesh.centroid
    n, k = len(c), 2 * np.pi

    def jitter():
        return noise * rng.uniform(-1, 1, n)

    rho = 1 + 0.2 * np.sin(k * c[:, 0]) + jitter()
    vx = 0.3 * np.sin(k * c[:, 1]) + jitter()
    vy = 0.2 * np.cos(k * c[:, 0]) + jitter()
    P = 1 + 0.2 * np.cos(k * (c[:, 0] + c[:, 1])) + jitter()
    U = np.stack([rho, rho * vx, rho * vy, P / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy)], -1)
    return U * mesh.volume[:, None]


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


def voronoi_invariants(m, tol=1e-11):
    """Geometric properties every periodic Voronoi mesh has, independent of how it was built: the volumes tile the box;
    each cell's outward area vectors close; each face lies on the bisector plane of its two generators (its centroid
    equidistant from both, its area vector along their separation); each cell's volume is a third of the flux of the
    position through its faces (divergence theorem, 3D; half in 2D)."""
    N, F, D = m.n_cells, m.n_faces, m.dim
    box = np.asarray(m.box, dtype=np.float64)[:D]
    assert np.isclose(m.volume.sum(), np.prod(box), rtol=0, atol=1e-12)
    S = np.zeros((N, D))
    np.add.at(S, m.owner, m.area)
    np.add.at(S, m.neighbour, -m.area)
    assert np.abs(S).max() < 1e-14
    d = m.positions[m.neighbour] - m.positions[m.owner]
    d -= box * np.round(d / box)
    c = m.face_centroid  # relative to the owner's generator
    r_o = np.linalg.norm(c, axis=1)
    r_j = np.linalg.norm(c - d, axis=1)
    assert np.max(np.abs(r_o - r_j) / np.linalg.norm(d, axis=1)) < tol
    a = np.linalg.norm(m.area, axis=1)
    keep = a > 1e-12 * a.max()
    cos = np.einsum("fk,fk->f", m.area[keep], d[keep]) / (a[keep] * np.linalg.norm(d[keep], axis=1))
    assert np.max(np.abs(cos - 1)) < 1e-9
    flux = np.einsum("fk,fk->f", m.area, c)  # A . x_f from the owner's generator
    V = np.zeros(N)
    np.add.at(V, m.owner, flux)
    np.add.at(V, m.neighbour, -np.einsum("fk,fk->f", m.area, c - d))
    assert np.max(np.abs(V / D - m.volume) / m.volume) < tol
