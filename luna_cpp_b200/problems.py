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


# ---- 1D lines (luna-cpp's src/hydro/problems_1d.hpp): cell averages of LUNA's setups on [a, b] -----------------------

def _conserved_1d(W, gamma):
    """problems_1d.hpp's conserved (:31-33), in its operation order."""
    return np.stack([W[0], W[0] * W[1], W[2] / (gamma - 1) + 0.5 * W[0] * W[1] * W[1]], axis=-1)


def _fraction_below(x, a, b):
    return np.clip((x - a) / (b - a), 0.0, 1.0)


def _tube(left, right, x0, gamma):
    """A jump at x0: exact cell averages by volume fraction (problems_1d.hpp:37-43)."""
    l = _conserved_1d(np.asarray(left, dtype=np.float64), gamma)
    r = _conserved_1d(np.asarray(right, dtype=np.float64), gamma)

    def average(a, b):
        f = _fraction_below(x0, a, b)[:, None]
        return f * l + (1 - f) * r

    return average


def _shock_into_wave(left, x0, amp, k, gamma):
    """A shock at x0 into 1 + amp sin(k x): exact cell averages (problems_1d.hpp:46-51)."""

    def average(a, b):
        h = b - a
        f = _fraction_below(x0, a, b)
        lo = np.maximum(a, x0)
        rho = f * left[0] + (1 - f)
        rho = np.where(b > lo, rho + amp * (np.cos(k * lo) - np.cos(k * b)) / k / h, rho)
        return np.stack([rho, f * left[0] * left[1],
                         f * (left[2] / (gamma - 1) + 0.5 * left[0] * left[1] * left[1]) + (1 - f) / (gamma - 1)], axis=-1)

    return average


def _woodward_colella(a, b):
    """Woodward-Colella's cell averages (problems_1d.hpp:55-60)."""
    f1, f2 = _fraction_below(0.1, a, b), _fraction_below(0.9, a, b)
    p = f1 * 1000 + (f2 - f1) * 0.01 + (1 - f2) * 100
    return np.stack([np.ones_like(p), np.zeros_like(p), p / (1.4 - 1)], axis=-1)


def line_problem(name: str) -> dict:
    """A 1D problem of problems_1d.hpp's table (:207-243): the line [origin, origin + L], its walls, t_end, gamma and
    ``average(a, b)``, the extensive-per-length conserved state of cells [a, b] (absolute coordinates, arrays)."""
    outflow, closed = ("outflow", "outflow"), ("reflective", "reflective")
    toro = {"sod": ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.25), "toro-1": ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.25),
            "toro-2": ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4), 0.15), "toro-3": ((1.0, 0.0, 1000.0), (1.0, 0.0, 0.01), 0.012),
            "toro-4": ((1.0, 0.0, 0.01), (1.0, 0.0, 100.0), 0.035),
            "toro-5": ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950), 0.035)}
    if name in toro:
        left, right, t_end = toro[name]
        return {"L": 1.0, "origin": 0.0, "t_end": t_end, "gamma": 1.4, "walls": outflow,
                "average": _tube(left, right, 0.5, 1.4)}
    if name == "shu-osher":
        # moving_walls (:287-298): gas enters supersonically at the left, so on a moving line that wall holds its state
        left = (3.857143, 2.629369, 10.33333)
        return {"L": 10.0, "origin": -5.0, "t_end": 1.8, "gamma": 1.4, "walls": outflow,
                "average": _shock_into_wave(left, -4.0, 0.2, 5.0, 1.4),
                "moving_walls": ("inflow", "outflow"), "moving_inflow": (left, (0.0, 0.0, 0.0))}
    if name == "woodward-colella":
        return {"L": 1.0, "origin": 0.0, "t_end": 0.038, "gamma": 1.4, "walls": closed, "average": _woodward_colella}
    raise ValueError(f"unknown 1D problem {name!r}")


def line_tube(left, right, t_end: float, x0: float = 0.5, gamma: float = 1.4, walls=("outflow", "outflow"), L: float = 1.0) -> dict:
    """A Riemann problem on [0, L] (problems_1d.hpp's tube, :37-43): primitives left of x0 and right of it."""
    return {"L": L, "origin": 0.0, "t_end": t_end, "gamma": gamma, "walls": tuple(walls), "average": _tube(left, right, x0, gamma)}


def line_keys(positions, L: float):
    """The generators of a line of length L on the 1D mesh's grid (step = L 2^-52, period 2^52 steps): sorted
    keys, the slot -> position order, the step and the period."""
    x = np.asarray(positions, dtype=np.float64)
    step = np.ldexp(L, -52)
    keys = np.rint(x / step).astype(np.int64)
    order = np.argsort(keys, kind="stable")
    return keys[order], order, float(step), 1 << 52


def line_state(problem: dict, keys, step: float) -> np.ndarray:
    """Q [n, 3] in slot order: each cell's average of the problem over its extent (midway to its neighbours, to a wall at
    the ends), as hydro1d_test.cpp's set() fills it (:40-55)."""
    k = np.asarray(keys, dtype=np.float64)
    gaps = np.concatenate([[2 * k[0]], np.diff(k), [2 * ((1 << 52) - k[-1])]])
    volume = (gaps[:-1] + gaps[1:]) * (0.5 * step)
    centroid = (gaps[1:] - gaps[:-1]) * (0.25 * step)
    x = k * step
    a = x + centroid - 0.5 * volume
    b = x + centroid + 0.5 * volume
    U = problem["average"](a + problem["origin"], b + problem["origin"])
    return U * (b - a)[:, None]
