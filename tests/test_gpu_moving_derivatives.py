"""The moving step's derivatives at fixed topology, orders 0 and 1 (luna_fv_step_moving_tangent[_end] /
luna_fv_step_moving_adjoint[_begin, _new_mesh], the reference's step_moving_tangent / step_moving_adjoint,
finite_volume.hpp:2431-3155) on 2D meshes, with the 2D
geometry derivative of luna_cpp_b200/geometry_derivative.py: the adjoint is the tangent's transpose over several steps
(the dot test), and the tangent equals central differences of the forward step (the same dt, the host remesh), as the
reference's derivative tests check theirs (hydro_derivatives_test.cpp:592-716)."""
import numpy as np
import pytest

from conftest import jittered_mesh
from luna_cpp_b200 import hydro
from luna_cpp_b200.geometry_derivative import Geometry2D
from luna_cpp_b200.mesh import build_mesh

pytestmark = pytest.mark.gpu

GAMMA = 5.0 / 3.0


def shear_state(mesh, seed=4):
    """A smooth 2D shear layer with a transverse wave and a little seeded noise (no limiter ties), extensive."""
    x = mesh.positions
    rng = np.random.default_rng(seed)
    layer = np.tanh((0.25 - np.abs(x[:, 1] - 0.5)) / 0.08)
    rho = 1.5 + 0.5 * layer + 1e-3 * rng.uniform(-1, 1, len(x))
    vx = 0.4 * layer
    vy = 0.05 * np.sin(2 * np.pi * x[:, 0])
    P = 2.5 + 0.1 * np.cos(2 * np.pi * x[:, 1])
    U = np.stack([rho, rho * vx, rho * vy, P / (GAMMA - 1) + 0.5 * rho * (vx * vx + vy * vy)], -1)
    return U * mesh.volume[:, None]


class Run:
    """Moving steps from (Q, x): the forward through the library with the host remesh; the tangent and the adjoint with
    the 2D geometry derivative of each mesh they read (order 1: the step runs inside them, between their passes)."""

    def __init__(self, mesh, riemann="hllc", order=0):
        self.box = tuple(mesh.box[:2])
        self.riemann = riemann
        self.fv = hydro.FiniteVolume(mesh, hydro.Gas(GAMMA), order=order, motion="moving", riemann=riemann)

    def remesh(self, p):
        return build_mesh(p, box=self.box)

    def start(self, q, x):
        self.fv.set_mesh(build_mesh(x, box=self.box))
        self.fv.set_state(q)

    def forward(self, q, x, dts):
        self.start(q, x)
        path = []
        for dt in dts:
            path.append((self.fv.get_state(), self.fv.positions()))
            self.fv.time_step(0.3)  # the sweep: the point velocities of this state
            self.fv.step_moving(dt, lambda p: build_mesh(p, box=self.box))
        return self.fv.get_state(), self.fv.positions(), path

    def tangent(self, q, x, dq, dx, dts):
        self.start(q, x)
        for dt in dts:
            self.fv.time_step(0.3)
            dq, dx = self.fv.step_moving_tangent(dt, dq, dx, Geometry2D, self.remesh)  # the step runs inside
        return dq, dx

    def adjoint(self, path, qbar, xbar, dts):
        for (q, x), dt in zip(reversed(path), reversed(dts)):
            self.start(q, x)
            self.fv.time_step(0.3)
            qbar, xbar = self.fv.step_moving_adjoint(dt, qbar, xbar, Geometry2D, self.remesh)
        return qbar, xbar


def base(n=24, seed=2):
    mesh = jittered_mesh(n, dim=2, jitter=0.3, seed=seed)
    return mesh, shear_state(mesh)


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("riemann", ["hllc", "hll"])
def test_moving_dot_test(cuda, riemann, order):
    """<qbar, J dq> + <xbar, J dx> = <J^T qbar, dq> + <J^T xbar, dx> over 3 steps, relative to the sum of the products'
    magnitudes: 1e-12 (the reference's C1, hydro_derivatives_test.cpp:595); order 0, and order 1 (two passes on the
    meshes of t^n and t^n+1, the limited fit's derivative in W and in the geometry)."""
    mesh, q0 = base()
    run = Run(mesh, riemann, order)
    x0 = mesh.positions.copy()
    run.start(q0, x0)
    dts = [0.5 * run.fv.time_step(0.3)] * 3
    qN, xN, path = run.forward(q0, x0, dts)
    rng = np.random.default_rng(7)
    dq = rng.normal(size=q0.shape) * np.abs(q0)
    dx = rng.normal(size=x0.shape) * 1e-3
    Jq, Jx = run.tangent(q0, x0, dq, dx, dts)
    qbar, xbar = rng.normal(size=q0.shape), rng.normal(size=x0.shape)
    Tq, Tx = run.adjoint(path, qbar, xbar, dts)
    lhs = float(np.sum(qbar * Jq) + np.sum(xbar * Jx))
    rhs = float(np.sum(Tq * dq) + np.sum(Tx * dx))
    size = float(np.sum(np.abs(qbar * Jq)) + np.sum(np.abs(xbar * Jx)) + np.sum(np.abs(Tq * dq)) + np.sum(np.abs(Tx * dx)))
    assert abs(lhs - rhs) < 1e-12 * size, (lhs, rhs, size)


@pytest.mark.parametrize("order", [0, 1])
def test_moving_dot_test_3d(cuda, order):
    """The 3D kernels: the dot test over two steps on 8^3 jittered generators with the reference's 3D wave state and a
    null geometry derivative (the same linear map on both sides), 1e-12 of the products' magnitudes."""
    from conftest import wave_state_3d
    from luna_cpp_b200.geometry_derivative import NullGeometry

    mesh = jittered_mesh(8, dim=3, jitter=0.15, seed=4)
    q0 = wave_state_3d(mesh)
    box = tuple(mesh.box[:3])
    fv = hydro.FiniteVolume(mesh, hydro.Gas(GAMMA), order=order, motion="moving")
    remesh = lambda p: build_mesh(p, box=box)  # noqa: E731
    x0 = mesh.positions.copy()

    def start(q, x):
        fv.set_mesh(build_mesh(x, box=box))
        fv.set_state(q)

    start(q0, x0)
    dts = [0.5 * fv.time_step(0.3)] * 2
    path = []
    for dt in dts:
        path.append((fv.get_state(), fv.positions()))
        fv.time_step(0.3)
        fv.step_moving(dt, remesh)
    rng = np.random.default_rng(8)
    dq0, dx0 = rng.normal(size=q0.shape) * np.abs(q0), rng.normal(size=x0.shape) * 1e-3
    start(q0, x0)
    dq, dx = dq0, dx0
    for dt in dts:
        fv.time_step(0.3)
        dq, dx = fv.step_moving_tangent(dt, dq, dx, NullGeometry, remesh)
    qbar, xbar = rng.normal(size=q0.shape), rng.normal(size=x0.shape)
    Tq, Tx = qbar, xbar
    for (q, x), dt in zip(reversed(path), reversed(dts)):
        start(q, x)
        fv.time_step(0.3)
        Tq, Tx = fv.step_moving_adjoint(dt, Tq, Tx, NullGeometry, remesh)
    lhs = float(np.sum(qbar * dq) + np.sum(xbar * dx))
    rhs = float(np.sum(Tq * dq0) + np.sum(Tx * dx0))
    size = float(np.sum(np.abs(qbar * dq)) + np.sum(np.abs(xbar * dx)) + np.sum(np.abs(Tq * dq0)) + np.sum(np.abs(Tx * dx0)))
    assert abs(lhs - rhs) < 1e-12 * size, (lhs, rhs, size)


def test_moving_tangent_equals_central_differences(cuda):
    """J (dq, dx) over 2 steps against central differences of the forward (the same dt, each side its own host remesh,
    the starting meshes' topology fixed within +- h): within 1e-6 of each block's largest entry at h = 1e-6 (dq relative
    to |Q|, dx of 1e-3 cell widths)."""
    mesh, q0 = base(seed=5)
    run = Run(mesh)
    x0 = mesh.positions.copy()
    run.start(q0, x0)
    dts = [0.5 * run.fv.time_step(0.3)] * 2
    rng = np.random.default_rng(3)
    dq = rng.normal(size=q0.shape) * np.abs(q0)
    dx = rng.normal(size=x0.shape) / 24
    Jq, Jx = run.tangent(q0, x0, dq, dx, dts)
    h = 1e-6
    qp, xp, _ = run.forward(q0 + h * dq, x0 + h * dx, dts)
    qm, xm, _ = run.forward(q0 - h * dq, x0 - h * dx, dts)
    box = np.array(mesh.box[:2])
    fq = (qp - qm) / (2 * h)
    dxm = xp - xm
    fx = (dxm - box * np.round(dxm / box)) / (2 * h)  # the drift wraps into the box
    assert np.max(np.abs(Jq - fq)) <= 1e-6 * np.max(np.abs(fq))
    assert np.max(np.abs(Jx - fx)) <= 1e-6 * np.max(np.abs(fx))


def test_moving_tangent_order_1_equals_central_differences(cuda):
    """Order 1 with the grid steps held (the reference's steps_fixed), one step along a Q direction of 1e-9 of each entry
    (dx = 0), as the reference's order-1 check (hydro_derivatives_test.cpp:1598-1655): J dq equals the central difference
    of the forward within 1e-5 of the largest entry, except next to a point whose grid step changed within +- h (the
    tangent holds it; there one side matches), at most 8 cells per such point."""
    mesh, q0 = base(seed=5)
    run = Run(mesh, order=1)
    run.fv.set_steps_fixed(True)
    x0 = mesh.positions.copy()
    run.start(q0, x0)
    dts = [0.5 * run.fv.time_step(0.3)]
    rng = np.random.default_rng(3)
    dq = rng.normal(size=q0.shape) * np.abs(q0)
    Jq, Jx = run.tangent(q0, x0, dq, np.zeros_like(x0), dts)
    assert np.all(Jx == 0)
    q_end = run.fv.get_state()  # the tangent's own forward
    h = 1e-9
    qp, xp, _ = run.forward(q0 + h * dq, x0, dts)
    qm, xm, _ = run.forward(q0 - h * dq, x0, dts)
    changed = int(np.sum(np.any(xp != xm, axis=1)))
    scale = np.max(np.abs(qp - qm)) / (2 * h)
    central = np.max(np.abs(Jq - (qp - qm) / (2 * h)), axis=1) / scale
    one_sided = np.minimum(np.max(np.abs(Jq - (qp - q_end) / h), axis=1), np.max(np.abs(Jq - (q_end - qm) / h), axis=1)) / scale
    off = central > 1e-5
    assert int(off.sum()) <= 8 * changed, (int(off.sum()), changed)
    assert np.all(one_sided[off] < 1e-5), float(np.max(one_sided[off]))


def test_moving_adjoint_states(cuda):
    """The last part of the order-1 adjoint refuses to run before its first two; the order-1 tangent needs a remesh."""
    mesh, q0 = base(8)
    fv = hydro.FiniteVolume(mesh, hydro.Gas(GAMMA), order=1, motion="moving")
    fv.set_state(q0)
    fv.time_step(0.3)
    with pytest.raises(hydro.LunaError):  # the last part without begin and the new mesh
        hydro.check(hydro.lib().luna_fv_step_moving_adjoint(fv.handle, 1e-3, np.zeros_like(q0).ctypes.data,
                                                             np.zeros((mesh.n_cells, 2)).ctypes.data, np.zeros(mesh.n_cells).ctypes.data,
                                                             np.zeros((mesh.n_cells, 2)).ctypes.data,
                                                             np.zeros((mesh.n_faces, 2)).ctypes.data,
                                                             np.zeros((mesh.n_faces, 2)).ctypes.data, 0))
    with pytest.raises(ValueError):
        fv.step_moving_tangent(1e-3, np.zeros_like(q0), np.zeros((mesh.n_cells, 2)), Geometry2D)
