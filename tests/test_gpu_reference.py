"""The CUDA path (through the C ABI) against the reference's own solver built on the CPU (oracle/_ref: luna-cpp's
finite_volume.hpp compiled unmodified against a host Kokkos), on the same meshes and states: the C-oracle parity
chain made direct, plus the one derivative the C oracle does not restate, step_tangent.

Tolerances are the parity bounds of the oracle tests: FP64 50 steps 1e-12 relative L1 per field, one step 1e-13
relative, the adjoint 1e-11 relative; the tangent, linearised at the same face states but with the GPU's multiply-add
contraction, 1e-10 relative (max norm)."""
import numpy as np
import pytest

from conftest import jittered_mesh
from luna_cpp_b200 import hydro
from luna_cpp_b200.mesh import build_mesh
from luna_cpp_b200.problems import point_blast, rough_state
from oracle import ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def reference(cuda):
    if not R.available():
        pytest.skip("the reference's CPU build (oracle/_ref) is not in this tree")
    return R


def rel_l1(a, b):
    return float(np.max(np.abs(a - b).sum(0) / np.maximum(np.abs(b).sum(0), 1e-300)))


def test_c0_point_blast_50_steps(reference):
    """32^3 jittered generators, the point blast, MUSCL-Hancock + HLLC, CFL 0.3, 50 steps, FP64, each side its own dt."""
    mesh = jittered_mesh(32)
    q0 = point_blast(mesh, radius_cells=2.0)
    gpu, ref = hydro.FiniteVolume(mesh), R.ReferenceFV(mesh)
    gpu.set_state(q0)
    ref.set_state(q0)
    for _ in range(50):
        dg, dr = gpu.time_step(0.3), ref.time_step(0.3)
        assert abs(dg - dr) <= 1e-13 * dr
        gpu.step(dg)
        ref.step(dr)
    assert rel_l1(gpu.get_state(), ref.get_state()) <= 1e-12


@pytest.mark.parametrize("precision,ref_precision,tol", [("grad32", "grad32", 1e-6), ("grad16", "grad16", 1e-5),
                                                          ("fp32", "riemann32", 1e-6)])
def test_precision_policies_one_step(reference, precision, ref_precision, tol):
    """The reduced policies against the reference running the same policy, one step (relative, max norm)."""
    mesh = jittered_mesh(16)
    q0 = point_blast(mesh, radius_cells=2.0)
    gpu, ref = hydro.FiniteVolume(mesh, precision=precision), R.ReferenceFV(mesh, precision=ref_precision)
    gpu.set_state(q0)
    ref.set_state(q0)
    dt = ref.time_step(0.3)
    gpu.time_step(0.3)
    gpu.step(dt)
    ref.step(dt)
    got, want = gpu.get_state(), ref.get_state()
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))


@pytest.mark.parametrize("dim", [3, 2])
def test_step_adjoint(reference, dim):
    mesh = jittered_mesh(12 if dim == 3 else 40, dim=dim)
    q0 = rough_state(mesh.n_cells, dim=dim) * mesh.volume[:, None]
    qbar = np.random.default_rng(9).standard_normal(q0.shape)
    gpu, ref = hydro.FiniteVolume(mesh), R.ReferenceFV(mesh)
    gpu.set_state(q0)
    ref.set_state(q0)
    dt = ref.time_step(0.3)
    got, want = gpu.step_adjoint(dt, qbar), ref.step_adjoint(dt, qbar)
    assert np.max(np.abs(got - want)) <= 1e-11 * np.max(np.abs(want))


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("limiter", ["face_centroid", "none"])
def test_step_tangent(reference, dim, limiter):
    """step_tangent (finite_volume.hpp:2033-2062) after time_step: J dq and the state it advances."""
    mesh = jittered_mesh(12 if dim == 3 else 40, dim=dim)
    q0 = rough_state(mesh.n_cells, dim=dim) * mesh.volume[:, None]
    dq = np.random.default_rng(dim).standard_normal(q0.shape) * np.abs(q0)
    gpu, ref = hydro.FiniteVolume(mesh, limiter=limiter), R.ReferenceFV(mesh, limiter=limiter)
    gpu.set_state(q0)
    ref.set_state(q0)
    dt = ref.time_step(0.3)
    assert abs(gpu.time_step(0.3) - dt) <= 1e-14 * dt
    got, want = gpu.step_tangent(dt, dq), ref.step_tangent(dt, dq)
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))
    assert np.max(np.abs(gpu.get_state() - ref.get_state())) <= 1e-13 * np.max(np.abs(ref.get_state()))


def test_moving_steps(reference):
    """Three moving steps of the blast on 16^3 jittered generators: the reference remeshes through its mesh update,
    the GPU path through the caller's remesh between its two flux passes."""
    mesh = jittered_mesh(16)
    q0 = point_blast(mesh, radius_cells=2.0)
    box = tuple(mesh.box[:3])
    gpu = hydro.FiniteVolume(mesh, motion="moving")
    ref = R.ReferenceFV(mesh, moving=True, remesh=lambda x: build_mesh(x, box=box))
    gpu.set_state(q0)
    ref.set_state(q0)
    for _ in range(3):
        dg, dr = gpu.time_step(0.3), ref.time_step(0.3)
        assert abs(dg - dr) <= 1e-13 * dr
        gpu.step_moving(dr, lambda x: build_mesh(x, box=box))
        ref.step(dr)
    assert np.array_equal(gpu.positions(), ref.positions())
    got, want = gpu.get_state(), ref.get_state()
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


@pytest.mark.parametrize("precision,ref_precision", [("fp32", "riemann32"), ("single", "single")])
def test_moving_step_float_policies(reference, precision, ref_precision):
    """One moving step of the blast on 16^3 jittered generators in the float policies the moving configuration runs
    (riemann32: the Riemann solve in float; single: the gradients, face states, solve and flux rows in float) against the
    reference running the same policy: the same positions, Q within 1e-5 of the largest (float face arithmetic)."""
    mesh = jittered_mesh(16)
    q0 = point_blast(mesh, radius_cells=2.0)
    box = tuple(mesh.box[:3])
    gpu = hydro.FiniteVolume(mesh, motion="moving", precision=precision)
    ref = R.ReferenceFV(mesh, moving=True, precision=ref_precision, remesh=lambda x: build_mesh(x, box=box))
    gpu.set_state(q0)
    ref.set_state(q0)
    dg, dr = gpu.time_step(0.3), ref.time_step(0.3)
    assert abs(dg - dr) <= 1e-6 * dr
    gpu.step_moving(dr, lambda x: build_mesh(x, box=box))
    ref.step(dr)
    assert np.array_equal(gpu.positions(), ref.positions())
    got, want = gpu.get_state(), ref.get_state()
    assert np.max(np.abs(got - want)) <= 1e-5 * np.max(np.abs(want))


@pytest.mark.parametrize("dim", [2, 3])
def test_moving_steps_order_0(reference, dim):
    """The order-0 moving step (step(): FaceFlux<0, true> on the current mesh with the point velocities' face velocities,
    then move() off the grid and the mesh update, finite_volume.hpp:205-226, :1212-1228): three steps against the
    reference's own, each side remeshing with the host builder."""
    from luna_cpp_b200.problems import rough_state

    mesh = jittered_mesh(24 if dim == 2 else 12, dim=dim, jitter=0.3 if dim == 2 else 0.1)
    q0 = rough_state(mesh.n_cells, dim=dim) * mesh.volume[:, None]
    box = tuple(mesh.box[:dim])
    gpu = hydro.FiniteVolume(mesh, order=0, motion="moving")
    ref = R.ReferenceFV(mesh, order=0, moving=True, remesh=lambda x: build_mesh(x, box=box))
    gpu.set_state(q0)
    ref.set_state(q0)
    for _ in range(3):
        dg, dr = gpu.time_step(0.3), ref.time_step(0.3)
        assert abs(dg - dr) <= 1e-13 * dr
        gpu.step_moving(dr, lambda x: build_mesh(x, box=box))
        ref.step(dr)
    assert np.max(np.abs(gpu.positions() - ref.positions())) <= 1e-15
    got, want = gpu.get_state(), ref.get_state()
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


@pytest.mark.parametrize("riemann", ["hllc", "hll"])
def test_moving_derivatives_order_0(reference, riemann):
    """The GPU's order-0 moving tangent and adjoint against the reference's own step_moving_tangent /
    step_moving_adjoint (finite_volume.hpp:2431-2604) on a 2D shear layer, both with this repository's 2D geometry
    derivative: J (dq, dx) and J^T (qbar, xbar) within 1e-10 of the largest entry."""
    from luna_cpp_b200.geometry_derivative import Geometry2D

    mesh = jittered_mesh(24, dim=2, jitter=0.3, seed=2)
    x0 = mesh.positions.copy()
    layer = np.tanh((0.25 - np.abs(x0[:, 1] - 0.5)) / 0.08)
    rho, vx, vy = 1.5 + 0.5 * layer, 0.4 * layer, 0.05 * np.sin(2 * np.pi * x0[:, 0])
    q0 = np.stack([rho, rho * vx, rho * vy, 2.5 / (2 / 3) + 0.5 * rho * (vx * vx + vy * vy)], -1) * mesh.volume[:, None]
    remesh = lambda p: build_mesh(p, box=(1.0, 1.0))  # noqa: E731
    gpu = hydro.FiniteVolume(mesh, hydro.Gas(5.0 / 3.0), order=0, motion="moving", riemann=riemann)
    ref = R.ReferenceFV(mesh, gamma=5.0 / 3.0, order=0, moving=True, riemann=riemann, remesh=remesh)
    gpu.set_state(q0)
    ref.set_state(q0)
    dt = 0.5 * ref.time_step(0.3)
    gpu.time_step(0.3)
    rng = np.random.default_rng(5)
    dq, dx = rng.normal(size=q0.shape) * np.abs(q0), rng.normal(size=x0.shape) * 1e-3
    got = gpu.step_moving_tangent(dt, dq, dx, Geometry2D(gpu.mesh))
    want = ref.step_moving_tangent(dt, dq, dx, Geometry2D(ref.mesh))
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))
    ref.set_positions(x0)
    ref.set_state(q0)
    ref.time_step(0.3)
    qb, xb = rng.normal(size=q0.shape), rng.normal(size=x0.shape)
    got = gpu.step_moving_adjoint(dt, qb, xb, Geometry2D(gpu.mesh))
    want = ref.step_moving_adjoint(dt, qb, xb, Geometry2D(ref.mesh))
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))


@pytest.mark.parametrize("steps_fixed", [False, True])
@pytest.mark.parametrize("riemann", ["hllc", "hll"])
def test_moving_derivatives_order_1(reference, riemann, steps_fixed):
    """The GPU's order-1 moving tangent and adjoint (two passes around the step, the limited fit's derivative in W and in
    the geometry of both meshes) against the reference's own step_moving_tangent / step_moving_adjoint
    (finite_volume.hpp:2767-3155), with the grid steps' derivative (dw-hat = dw) and with them held (steps_fixed), on the
    reference's own wave state (every field non-uniform: a uniform one leaves the limiter's scale to rounding), both with
    this repository's 2D geometry derivative of each mesh: J (dq, dx) and J^T (qbar, xbar) within 1e-9 of the largest
    entry."""
    from conftest import wave_state_2d
    from luna_cpp_b200.geometry_derivative import Geometry2D

    mesh = jittered_mesh(24, dim=2, jitter=0.3, seed=2)
    x0 = mesh.positions.copy()
    q0 = wave_state_2d(mesh)
    remesh = lambda p: build_mesh(p, box=(1.0, 1.0))  # noqa: E731
    gpu = hydro.FiniteVolume(mesh, hydro.Gas(5.0 / 3.0), order=1, motion="moving", riemann=riemann)
    gpu.set_steps_fixed(steps_fixed)
    ref = R.ReferenceFV(mesh, gamma=5.0 / 3.0, order=1, moving=True, riemann=riemann, remesh=remesh)
    gpu.set_state(q0)
    ref.set_state(q0)
    dt = 0.5 * ref.time_step(0.3)
    gpu.time_step(0.3)
    rng = np.random.default_rng(5)
    dq, dx = rng.normal(size=q0.shape) * np.abs(q0), rng.normal(size=x0.shape) * 1e-3
    got = gpu.step_moving_tangent(dt, dq, dx, Geometry2D, remesh)
    want = ref.step_moving_tangent(dt, dq, dx, Geometry2D, steps_fixed=steps_fixed)
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))
    gpu.set_mesh(mesh)
    gpu.set_state(q0)
    gpu.time_step(0.3)
    ref.set_positions(x0)
    ref.set_state(q0)
    ref.time_step(0.3)
    qb, xb = rng.normal(size=q0.shape), rng.normal(size=x0.shape)
    got = gpu.step_moving_adjoint(dt, qb, xb, Geometry2D, remesh)
    want = ref.step_moving_adjoint(dt, qb, xb, Geometry2D, steps_fixed=steps_fixed)
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))


@pytest.mark.parametrize("order", [0, 1])
def test_moving_derivatives_3d_null_geometry(reference, order):
    """The moving derivatives' kernels in 3D (dimension-generic; no 3D geometry derivative here, voronoi-cpp's
    MeshDerivative being absent): with a null geometry derivative on both sides (V, c, A, x_f held; the reference's cost
    test does the same), the GPU's tangent and adjoint of one moving step against the reference's own on 8^3 jittered
    generators and the reference's 3D wave state (hydro_derivatives_test.cpp:1513-1516): within 1e-9 of the largest
    entry, orders 0 and 1."""
    from conftest import wave_state_3d
    from luna_cpp_b200.geometry_derivative import NullGeometry

    mesh = jittered_mesh(8, dim=3, jitter=0.15, seed=4)
    x0 = mesh.positions.copy()
    q0 = wave_state_3d(mesh)
    remesh = lambda p: build_mesh(p, box=(1.0, 1.0, 1.0))  # noqa: E731
    gpu = hydro.FiniteVolume(mesh, hydro.Gas(5.0 / 3.0), order=order, motion="moving")
    ref = R.ReferenceFV(mesh, gamma=5.0 / 3.0, order=order, moving=True, remesh=remesh)
    gpu.set_state(q0)
    ref.set_state(q0)
    dt = 0.5 * ref.time_step(0.3)
    gpu.time_step(0.3)
    rng = np.random.default_rng(6)
    dq, dx = rng.normal(size=q0.shape) * np.abs(q0), rng.normal(size=x0.shape) * 1e-3
    got = gpu.step_moving_tangent(dt, dq, dx, NullGeometry, remesh if order == 1 else None)
    want = ref.step_moving_tangent(dt, dq, dx, NullGeometry)
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))
    gpu.set_mesh(mesh)
    gpu.set_state(q0)
    gpu.time_step(0.3)
    ref.set_positions(x0)
    ref.set_state(q0)
    ref.time_step(0.3)
    qb, xb = rng.normal(size=q0.shape), rng.normal(size=x0.shape)
    got = gpu.step_moving_adjoint(dt, qb, xb, NullGeometry, remesh if order == 1 else None)
    want = ref.step_moving_adjoint(dt, qb, xb, NullGeometry)
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))
