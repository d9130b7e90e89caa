"""The C oracle (oracle/luna_oracle.c) against the reference's own solver: luna-cpp's src/hydro/finite_volume.hpp,
euler.hpp and precision.hpp compiled unmodified on the CPU (oracle/Makefile: a host-only Kokkos with OpenMP and the
part of voronoi-cpp the solver reads, over this repository's mesh arrays). Both run on the same mesh and state; each
takes its own time steps. CPU only.

Both are compiled without multiply-add contraction, and every reduction the reference runs is a minimum or an integer
sum, so the C restatement is expected to give the reference's bits; the bounds below are the parity bounds the CUDA
path is held to against the oracle (1e-12 relative L1 over 50 steps, 1e-11 for the adjoint), and each test also
records whether the two agree bit for bit."""
import numpy as np
import pytest

from conftest import jittered_mesh, random_mesh
from luna_cpp_b200.mesh import build_mesh
from luna_cpp_b200.problems import point_blast
from oracle import oracle as O
from oracle import ref as R


@pytest.fixture(scope="module")
def reference():
    if not R.available():
        try:
            R.build()
        except Exception as e:  # noqa: BLE001
            pytest.skip(f"the reference's solver could not be built here: {e}")
    return R


def rel_l1(a, b):
    """Relative L1 per conserved field, the largest over the fields."""
    return max(np.sum(np.abs(a[:, v] - b[:, v])) / max(np.sum(np.abs(b[:, v])), 1e-300) for v in range(b.shape[1]))


def run_both(mesh, q0, steps, ref_kw=None, **kw):
    a = O.OracleFV(mesh, **kw)
    b = R.ReferenceFV(mesh, **(ref_kw or {}), **kw)
    a.set_state(q0)
    b.set_state(q0)
    dts = []
    for _ in range(steps):
        da, db = a.time_step(0.3), b.time_step(0.3)
        dts.append((da, db))
        a.step(da)
        b.step(db)
    return a, b, dts


def test_c0_point_blast_50_steps(reference):
    """The CPU-runnable configuration: 32^3 jittered generators, the point blast, MUSCL-Hancock + HLLC, CFL 0.3,
    50 steps, FP64: the same 50 time steps and the same state (1e-12 relative L1 per field; bit-equal observed)."""
    mesh = jittered_mesh(32)
    q0 = point_blast(mesh, radius_cells=2.0)
    a, b, dts = run_both(mesh, q0, 50)
    for da, db in dts:
        assert abs(da - db) <= 1e-14 * db
    qa, qb = a.get_state(), b.get_state()
    assert rel_l1(qa, qb) <= 1e-12
    assert a.fallbacks() == b.fallbacks()
    assert np.array_equal(qa, qb) and all(da == db for da, db in dts), "bit-equal to the reference"


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("kw", [dict(riemann="hll"), dict(order=0), dict(per_face=False), dict(limiter="none"),
                                dict(order=0, per_face=False)],
                         ids=["hll", "order0", "per_cell", "no_limiter", "order0_per_cell"])
def test_variants(reference, dim, kw):
    """Every option of the constructor (finite_volume.hpp:79-107) on a jittered and a uniform random mesh, 6 steps."""
    for mesh in (jittered_mesh(10 if dim == 3 else 24, dim=dim), random_mesh(800 if dim == 3 else 500, dim=dim)):
        q0 = point_blast(mesh, radius_cells=2.0)
        a, b, dts = run_both(mesh, q0, 6, **kw)
        assert all(abs(da - db) <= 1e-14 * db for da, db in dts)
        assert rel_l1(a.get_state(), b.get_state()) <= 1e-13
        assert a.fallbacks() == b.fallbacks()
        assert np.array_equal(a.get_state(), b.get_state())


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("precision", ["grad32", "riemann32", "grad16", "single"])
def test_precision_policies(reference, dim, precision):
    """Grad32, riemann32 (Precision<double, float, double, float>) and Grad16 (binary16 gradient rows), 10 steps."""
    mesh = jittered_mesh(12 if dim == 3 else 32, dim=dim)
    q0 = point_blast(mesh, radius_cells=2.0)
    a, b, dts = run_both(mesh, q0, 10, precision=precision)
    assert all(abs(da - db) <= 1e-14 * db for da, db in dts)
    assert rel_l1(a.get_state(), b.get_state()) <= 1e-12
    assert np.array_equal(a.get_state(), b.get_state())


class _SharedRemesh:
    """Builds each new mesh once for both solvers: the second request for the same generators reuses it."""

    def __init__(self, box):
        self.box = box
        self.last = None

    def __call__(self, x):
        key = np.ascontiguousarray(x).tobytes()
        if self.last is None or self.last[0] != key:
            self.last = (key, build_mesh(x, box=self.box))
        return self.last[1]


@pytest.mark.parametrize("dim,nx,steps", [(3, 32, 50), (2, 48, 50)])
def test_moving_point_blast(reference, dim, nx, steps):
    """The moving step (step_moving, finite_volume.hpp:1497-1519: snapped generators, fluxes on the old and the new
    mesh, AREPO's regularisation), the blast over 50 steps: the same time steps, positions and state."""
    mesh = jittered_mesh(nx, dim=dim)
    q0 = point_blast(mesh, radius_cells=2.0)
    remesh = _SharedRemesh(tuple(mesh.box[:dim]))
    a = O.OracleFV(mesh, moving=True)
    b = R.ReferenceFV(mesh, moving=True, remesh=remesh)
    a.set_state(q0)
    b.set_state(q0)
    for _ in range(steps):
        da, db = a.time_step(0.3), b.time_step(0.3)
        assert abs(da - db) <= 1e-14 * db
        a.step_moving(da, remesh)
        b.step(db)
    qa, qb = a.get_state(), b.get_state()
    assert rel_l1(qa, qb) <= 1e-12
    assert np.array_equal(a.mesh.positions, b.positions())
    assert np.array_equal(qa, qb)


@pytest.mark.parametrize("dim,nx", [(3, 12), (2, 32)])
def test_step_adjoint(reference, dim, nx):
    """step_adjoint (finite_volume.hpp:2201-2231) at the state after 3 steps, a random Q bar: within 1e-11."""
    mesh = jittered_mesh(nx, dim=dim)
    q0 = point_blast(mesh, radius_cells=2.0)
    a, b, _ = run_both(mesh, q0, 3)
    dt = a.time_step(0.3)
    assert dt == b.time_step(0.3)
    qbar = np.random.default_rng(4).standard_normal(q0.shape)
    ga, gb = a.step_adjoint(dt, qbar), b.step_adjoint(dt, qbar)
    assert np.max(np.abs(ga - gb)) <= 1e-11 * np.max(np.abs(gb))
    assert np.array_equal(ga, gb)


def _shear(mesh, gamma=5.0 / 3.0):
    x = mesh.positions
    layer = np.tanh((0.25 - np.abs(x[:, 1] - 0.5)) / 0.08)
    rho = 1.5 + 0.5 * layer + 1e-3 * np.random.default_rng(4).uniform(-1, 1, len(x))
    vx, vy, P = 0.4 * layer, 0.05 * np.sin(2 * np.pi * x[:, 0]), 2.5 + 0.1 * np.cos(2 * np.pi * x[:, 1])
    U = np.stack([rho, rho * vx, rho * vy, P / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy)], -1)
    return U * mesh.volume[:, None]


def test_reference_moving_derivatives_dot_test(reference):
    """The reference's own step_moving_tangent / step_moving_adjoint (order 0, 2D) with this repository's 2D geometry
    derivative as their GeometryDerivative: the dot test to 1e-12 (the reference's C1, hydro_derivatives_test.cpp:595),
    which pins the geometry derivative's interface (tangent and adjoint, the adjoint adding to x's bar) to the reference's
    use of it."""
    from luna_cpp_b200.geometry_derivative import Geometry2D

    mesh = jittered_mesh(16, dim=2, jitter=0.3, seed=2)
    q0, x0 = _shear(mesh), mesh.positions.copy()
    ref = R.ReferenceFV(mesh, gamma=5.0 / 3.0, order=0, moving=True, remesh=lambda p: build_mesh(p, box=(1.0, 1.0)))
    ref.set_state(q0)
    dt = 0.5 * ref.time_step(0.3)
    rng = np.random.default_rng(1)
    dq, dx = rng.normal(size=q0.shape) * np.abs(q0), rng.normal(size=x0.shape) * 1e-3
    Jq, Jx = ref.step_moving_tangent(dt, dq, dx, Geometry2D(ref.mesh))
    ref.set_positions(x0)
    ref.set_state(q0)
    ref.time_step(0.3)
    qb, xb = rng.normal(size=q0.shape), rng.normal(size=x0.shape)
    Tq, Tx = ref.step_moving_adjoint(dt, qb, xb, Geometry2D(ref.mesh))
    lhs, rhs = np.sum(qb * Jq) + np.sum(xb * Jx), np.sum(Tq * dq) + np.sum(Tx * dx)
    size = np.sum(np.abs(qb * Jq)) + np.sum(np.abs(xb * Jx)) + np.sum(np.abs(Tq * dq)) + np.sum(np.abs(Tx * dx))
    assert abs(lhs - rhs) < 1e-12 * size
