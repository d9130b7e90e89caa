"""The order-0 moving step's derivatives at fixed topology (luna_fv_step_moving_tangent / luna_fv_step_moving_adjoint,
the reference's step_moving_tangent / step_moving_adjoint, finite_volume.hpp:2431-2604) on 2D meshes, with the 2D
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
    """Order-0 moving steps from (Q, x): the forward through the library with the host remesh; the tangent and the
    adjoint with the 2D geometry derivative of each step's starting mesh."""

    def __init__(self, mesh, riemann="hllc"):
        self.box = tuple(mesh.box[:2])
        self.riemann = riemann
        self.fv = hydro.FiniteVolume(mesh, hydro.Gas(GAMMA), order=0, motion="moving", riemann=riemann)

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
            dq, dx = self.fv.step_moving_tangent(dt, dq, dx, Geometry2D(self.fv.mesh))
            self.fv.step_moving(dt, lambda p: build_mesh(p, box=self.box))
        return dq, dx

    def adjoint(self, path, qbar, xbar, dts):
        for (q, x), dt in zip(reversed(path), reversed(dts)):
            self.start(q, x)
            self.fv.time_step(0.3)
            qbar, xbar = self.fv.step_moving_adjoint(dt, qbar, xbar, Geometry2D(self.fv.mesh))
        return qbar, xbar


def base(n=24, seed=2):
    mesh = jittered_mesh(n, dim=2, jitter=0.3, seed=seed)
    return mesh, shear_state(mesh)


@pytest.mark.parametrize("riemann", ["hllc", "hll"])
def test_moving_dot_test(cuda, riemann):
    """<qbar, J dq> + <xbar, J dx> = <J^T qbar, dq> + <J^T xbar, dx> over 3 steps, relative to the sum of the products'
    magnitudes: 1e-12 (the reference's C1, hydro_derivatives_test.cpp:595)."""
    mesh, q0 = base()
    run = Run(mesh, riemann)
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


def test_moving_derivatives_need_order_0(cuda):
    mesh, q0 = base(8)
    fv = hydro.FiniteVolume(mesh, hydro.Gas(GAMMA), order=1, motion="moving")
    fv.set_state(q0)
    with pytest.raises(hydro.LunaError):
        fv.step_moving_tangent(1e-3, np.zeros_like(q0), np.zeros((mesh.n_cells, 2)), Geometry2D(mesh))
