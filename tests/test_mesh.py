"""The periodic Voronoi builder emits voronoi-cpp's layout: CPU only."""
import numpy as np
import pytest

from conftest import jittered_mesh, random_mesh, voronoi_invariants
from luna_cpp_b200.mesh import build_mesh, jittered_points


@pytest.mark.parametrize("mesh_fn", [lambda: jittered_mesh(16), lambda: random_mesh(4096), lambda: jittered_mesh(32, 2)])
def test_layout_and_closure(mesh_fn):
    m = mesh_fn()
    N, F, D = m.n_cells, m.n_faces, m.dim
    assert np.isclose(m.volume.sum(), 1.0, rtol=0, atol=1e-12)
    assert (m.volume > 0).all()
    # Every cell's outward area vectors close (the discrete divergence of a constant vanishes).
    S = np.zeros((N, D))
    np.add.at(S, m.owner, m.area)
    np.add.at(S, m.neighbour, -m.area)
    assert np.abs(S).max() < 1e-14
    # Lists: each face appears once owned (f) in its owner's list and once as ~f in its neighbour's.
    assert m.cell_face_start[0] == 0 and m.cell_face_start[-1] == 2 * F
    for i in range(0, N, max(1, N // 97)):
        entries = m.cell_face[m.cell_face_start[i]:m.cell_face_start[i + 1]]
        for e in entries:
            f = e if e >= 0 else ~e
            if e >= 0:
                assert m.owner[f] == i
            else:
                assert m.neighbour[f] == i
    assert (m.owner < m.neighbour).all()
    assert m.inconsistent == 0


def test_face_count_matches_reference_ratio():
    """F/N = 7.95 on a jittered (0.1) 3D lattice, as the reference measures (README.md:301)."""
    m = jittered_mesh(32)
    assert abs(m.n_faces / m.n_cells - 7.95) < 0.05


def test_jittered_points_law():
    p = jittered_points((4, 4, 4), jitter=0.1, seed=1)
    h = 0.25
    lattice = (np.stack(np.meshgrid(np.arange(4), np.arange(4), np.arange(4), indexing="ij"), -1).reshape(-1, 3) + 0.5) * h
    d = (p - lattice + 0.5) % 1.0 - 0.5
    assert np.abs(d).max() <= 0.1 * h + 1e-15
    assert np.array_equal(p, jittered_points((4, 4, 4), jitter=0.1, seed=1))


def test_too_small_box_is_an_error():
    with pytest.raises(ValueError):
        build_mesh(np.array([[0.5, 0.5, 0.5], [0.1, 0.1, 0.1]]))


def hollow_points(nx=20, hole=0.36):
    """A jittered lattice with a hole of radius ``hole`` around the box centre and one generator at the centre: the
    centre cell reaches several times farther than the grid's sorted offsets."""
    p = jittered_points((nx, nx, nx), jitter=0.1, seed=4)
    keep = np.linalg.norm(p - 0.5, axis=1) > hole
    return np.concatenate([[[0.5, 0.5, 0.5]], p[keep]])


def test_cell_far_larger_than_the_spacing():
    """The search continues past the grid's offsets over the cube of buckets that can hold a cutting image: the centre
    cell of a hollow lattice is a closed polyhedron of the hole's size; volumes tile the box."""
    m = build_mesh(hollow_points())
    assert np.isclose(m.volume.sum(), 1.0, rtol=0, atol=1e-12)
    S = np.zeros((m.n_cells, 3))
    np.add.at(S, m.owner, m.area)
    np.add.at(S, m.neighbour, -m.area)
    assert np.abs(S).max() < 1e-14
    r = 0.36 / 2  # the centre cell holds at least the ball of half the hole's radius
    assert m.volume[0] > 4.0 / 3.0 * np.pi * r ** 3
    assert m.cell_face_start[1] - m.cell_face_start[0] > 30


def test_threads_do_not_change_the_mesh():
    """Cells are built independently and assembled in a fixed order: one thread and all threads give the same bytes."""
    p = jittered_points((14, 14, 14), jitter=0.1, seed=9)
    a, b = build_mesh(p, threads=1), build_mesh(p, threads=0)
    for f in ("owner", "neighbour", "cell_face_start", "cell_face", "area", "face_centroid", "centroid", "volume"):
        assert np.ascontiguousarray(getattr(a, f)).tobytes() == np.ascontiguousarray(getattr(b, f)).tobytes(), f


@pytest.mark.parametrize("mesh_fn", [lambda: jittered_mesh(16), lambda: random_mesh(4096), lambda: jittered_mesh(32, 2),
                                     lambda: build_mesh(hollow_points())])
def test_voronoi_invariants(mesh_fn):
    voronoi_invariants(mesh_fn())


def test_cell_far_larger_than_the_spacing_2d():
    """The far search in 2D: a jittered 40^2 lattice with a hole of radius 0.3 and one generator in its middle."""
    p = jittered_points((40, 40), jitter=0.1, seed=4)
    p = np.concatenate([[[0.5, 0.5]], p[np.linalg.norm(p - 0.5, axis=1) > 0.3]])
    m = build_mesh(p, box=(1.0, 1.0))
    voronoi_invariants(m)
    assert m.volume[0] > np.pi * 0.15 ** 2
