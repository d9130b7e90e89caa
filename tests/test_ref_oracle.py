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
