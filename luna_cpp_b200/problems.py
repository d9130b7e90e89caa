"""Initial states of the benchmark and test problems (primitive W per cell -> extensive Q = U(W) V).

- ``point_blast``: rho = 1, v = 0, p = 1e-5, with E deposited evenly by volume as thermal energy in the cells whose
  centroid lies within ``radius_cells`` mean cell widths of the box centre (the blast of the plain-method configuration);
- ``acoustic_wave``: background rho = 1, p = 3/5 (c = 1 at gamma 5/3), amplitude A sine along x, wavelength = box;
- ``shear_layer``: the 2D Kelvin-Helmholtz layer of the adjoint configuration;
- ``rough_state``: hydro_test.cpp's blast plus random perturbations (src/test/hydro_test.cpp:167-178) for invariants.
"""
from __future__ import annotations

import numpy as np


def conserved(W: np.ndarray, gamma: float) -> np.ndarray:
    """conserved(): W -> U (euler.hpp:165-172)."""
    W = np.asarray(W, dtype=np.float64)
    D = W.shape[-1] - 2
    rho = W[..., 0]
    v = W[..., 1:1 + D]
    kinetic = 0.5 * rho * np.sum(v * v, axis=-1)
    U = np.empty_like(W)
    U[..., 0] = rho
    U[..., 1:1 + D] = rho[..., None] * v
    U[..., D + 1] = W[..., D + 1] / (gamma - 1.0) + kinetic
    return U


def cell_centres(mesh) -> np.ndarray:
    """Absolute centroids (generator + centroid offset), wrapped into the box."""
    box = np.asarray(mesh.box, dtype=np.float64)
    c = mesh.positions + mesh.centroid
    return c - box * np.floor(c / box)


def point_blast(mesh, gamma=5.0 / 3.0, energy=1.0, radius_cells=2.0, p0=1e-5) -> np.ndarray:
    N, D = mesh.n_cells, mesh.dim
    box = np.asarray(mesh.box)
    h = (np.prod(box) / N) ** (1.0 / D)
    c = cell_centres(mesh)
    d = c - 0.5 * box
    r = np.sqrt(np.sum(d * d, axis=1))
    inside = r < radius_cells * h
    W = np.zeros((N, D + 2))
    W[:, 0] = 1.0
    W[:, D + 1] = p0
    U = conserved(W, gamma)
    Q = U * mesh.volume[:, None]
    vin = mesh.volume[inside].sum()
    # E spread evenly by volume: per unit volume E / vin added to the energy density of the inside cells.
    Q[inside, D + 1] += energy * mesh.volume[inside] / vin
    return Q


def acoustic_wave(mesh, gamma=5.0 / 3.0, amplitude=1e-6, p0=0.6) -> np.ndarray:
    N, D = mesh.n_cells, mesh.dim
    c = cell_centres(mesh)
    s = amplitude * np.sin(2.0 * np.pi * c[:, 0] / mesh.box[0])
    cs = np.sqrt(gamma * p0)
    W = np.zeros((N, D + 2))
    W[:, 0] = 1.0 + s
    W[:, 1] = cs * s
    W[:, D + 1] = p0 + gamma * p0 * s
    return conserved(W, gamma) * mesh.volume[:, None]


def shear_layer(mesh, coefficients, gamma=5.0 / 3.0) -> np.ndarray:
    c = cell_centres(mesh)
    x, y = c[:, 0], c[:, 1]
    inner = np.abs(y - 0.5) < 0.25
    W = np.zeros((mesh.n_cells, 4))
    W[:, 0] = np.where(inner, 2.0, 1.0)
    W[:, 1] = np.where(inner, 0.5, -0.5)
    k = np.arange(1, len(coefficients) + 1)
    W[:, 2] = 0.01 * np.sum(np.asarray(coefficients)[None, :] * np.sin(2 * np.pi * k[None, :] * x[:, None]), axis=1)
    W[:, 3] = 2.5
    return conserved(W, gamma) * mesh.volume[:, None]


def rough_state(n, dim=3, gamma=5.0 / 3.0, seed=11) -> np.ndarray:
    """Per unit volume: a blast in the first 8 cells plus uniform perturbations of every variable."""
    rng = np.random.default_rng(seed)
    W = np.empty((n, dim + 2))
    W[:, 0] = 1 + 0.3 * rng.uniform(-1, 1, n)
    for a in range(dim):
        W[:, 1 + a] = 0.5 * rng.uniform(-1, 1, n)
    W[:, dim + 1] = np.where(np.arange(n) < 8, 100.0, 1.0) * (1 + 0.3 * rng.uniform(-1, 1, n))
    return conserved(W, gamma)
