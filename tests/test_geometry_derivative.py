"""The 2D geometry derivative at fixed topology (luna_cpp_b200/geometry_derivative.py, the GeometryDerivative of
src/hydro/mesh_derivative.hpp:10-29 built as the reference's tests build theirs, src/test/reference_geometry_2d.hpp): its
circumcentre geometry equals the mesh builder's arrays, its tangent equals central differences of the mesh builder's
geometry under moved generators, and its adjoint is the tangent's transpose. On the CPU."""
import numpy as np
import pytest

from luna_cpp_b200.geometry_derivative import Geometry2D
from luna_cpp_b200.mesh import build_mesh, jittered_points


@pytest.fixture(scope="module")
def case():
    x = jittered_points((16, 16), jitter=0.3, seed=3)
    mesh = build_mesh(x, box=(1.0, 1.0))
    return mesh, Geometry2D(mesh)


def test_circumcentre_geometry_equals_the_mesh(case):
    mesh, G = case
    assert G.area_check < 1e-13 and G.centroid_check < 1e-13
    assert G.volume_check < 1e-13 and G.cell_centroid_check < 1e-13


def test_tangent_equals_central_differences(case):
    """h = 1e-6 along a random dx: the differences' O(h^2) error is 1e-8 of each quantity's largest derivative."""
    mesh, G = case
    dx = np.random.default_rng(1).normal(size=mesh.positions.shape)
    dV, dc, dA, dxf = G.tangent(dx)
    h = 1e-6
    plus = build_mesh(mesh.positions + h * dx, box=(1.0, 1.0))
    minus = build_mesh(mesh.positions - h * dx, box=(1.0, 1.0))
    assert np.array_equal(plus.owner, mesh.owner) and np.array_equal(minus.cell_face, mesh.cell_face)  # fixed topology
    for ours, name in ((dV, "volume"), (dc, "centroid"), (dA, "area"), (dxf, "face_centroid")):
        fd = (getattr(plus, name) - getattr(minus, name)) / (2 * h)
        assert np.max(np.abs(ours - fd)) <= 1e-6 * np.max(np.abs(fd)), name


def test_adjoint_is_the_transpose(case):
    mesh, G = case
    rng = np.random.default_rng(2)
    dx = rng.normal(size=mesh.positions.shape)
    t = G.tangent(dx)
    bars = [rng.normal(size=a.shape) for a in t]
    lhs = sum(float(np.sum(a * b)) for a, b in zip(t, bars))
    rhs = float(np.sum(G.adjoint(*bars) * dx))
    assert abs(lhs - rhs) <= 1e-13 * abs(lhs)


def test_refuses_3d(case):
    with pytest.raises(ValueError):
        Geometry2D(build_mesh(jittered_points((4, 4, 4), jitter=0.1, seed=1)))
