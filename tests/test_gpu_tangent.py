"""step_tangent (luna_fv_step_tangent): the dot test against the adjoint, central differences, the step it runs beside."""
import numpy as np
import pytest

from conftest import jittered_mesh
from luna_cpp_b200 import hydro
from luna_cpp_b200.problems import rough_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("riemann", ["hllc", "hll"])
@pytest.mark.parametrize("limiter", ["face_centroid", "none"])
def test_tangent_is_the_adjoints_transpose(cuda, dim, riemann, limiter):
    """The dot test (hydro_derivatives_test.cpp:380-400): <J dq, qbar> = <dq, J^T qbar> at the same state and dt, to
    1e-12, and the step beside the tangent leaves Q as step() does, bit for bit."""
    mesh = jittered_mesh(12 if dim == 3 else 40, dim=dim)
    V = dim + 2
    q0 = rough_state(mesh.n_cells, dim=dim) * mesh.volume[:, None]
    rng = np.random.default_rng(dim * 7 + (riemann == "hll") + 3 * (limiter == "none"))
    dq = rng.standard_normal((mesh.n_cells, V)) * np.abs(q0)
    qbar = rng.standard_normal((mesh.n_cells, V))
    fv = hydro.FiniteVolume(mesh, riemann=riemann, limiter=limiter)
    fv.set_state(q0)
    dt = fv.time_step(0.3)
    Jdq = fv.step_tangent(dt, dq)
    q_tangent = fv.get_state()
    fv.set_state(q0)
    JTqbar = fv.step_adjoint(dt, qbar)
    lhs, rhs = float((Jdq * qbar).sum()), float((dq * JTqbar).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))
    ref = hydro.FiniteVolume(mesh, riemann=riemann, limiter=limiter)
    ref.set_state(q0)
    ref.step(ref.time_step(0.3))
    assert np.array_equal(q_tangent, ref.get_state())


def test_tangent_matches_central_differences(cuda):
    """A smooth state on a jittered 2D mesh, three steps at a fixed dt: the tangent of the rollout against central
    differences of step() along the same direction (h = 1e-7), to 1e-6."""
    mesh = jittered_mesh(32, dim=2)
    c = mesh.positions + mesh.centroid
    X, Y = c[:, 0], c[:, 1]
    rho = 1.5 + 0.3 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    vx, vy = 0.2 * np.cos(2 * np.pi * Y), 0.1 * np.sin(2 * np.pi * X)
    P = 1.0 + 0.2 * np.cos(2 * np.pi * (X + Y))
    q0 = np.stack([rho, rho * vx, rho * vy, P / (2 / 3) + 0.5 * rho * (vx * vx + vy * vy)], 1) * mesh.volume[:, None]
    d = np.stack([np.sin(4 * np.pi * Y), 0 * X, np.cos(2 * np.pi * X), np.sin(2 * np.pi * (X - Y))], 1) * mesh.volume[:, None]
    fv = hydro.FiniteVolume(mesh)
    dt, steps, h = 2e-3, 3, 1e-7

    def rollout(q):
        fv.set_state(q)
        for _ in range(steps):
            fv.time_step(0.3)
            fv.step(dt)
        return fv.get_state()

    fv.set_state(q0)
    dq = d.copy()
    for _ in range(steps):
        fv.time_step(0.3)
        dq = fv.step_tangent(dt, dq)
    fd = (rollout(q0 + h * d) - rollout(q0 - h * d)) / (2 * h)
    assert np.max(np.abs(dq - fd)) <= 1e-6 * np.max(np.abs(fd))


def test_tangent_requires_fp64_static_order1(cuda):
    mesh = jittered_mesh(8)
    fv = hydro.FiniteVolume(mesh, precision="fp32")
    with pytest.raises(hydro.LunaError):
        fv.step_tangent(1e-3, np.zeros((mesh.n_cells, 5)))
