"""The device remesher (include/luna_remesh.h) and the sweep's tiles cut on the device.

The remesher clips each cell on the GPU with the host builder's code and assembles faces and lists in the host
builder's order, so its arrays equal ``build_mesh``'s bit for bit. A mesh given in device memory has its sweep tiles
cut on the device; the step's results do not depend on the tiling, so a step on it equals, bit for bit, the step on
the same mesh given in host memory (tiles cut on the host). A moving step with the remesh on the device equals the
moving step with the host remesh, bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest
from conftest import jittered_mesh, voronoi_invariants

from luna_cpp_b200 import hydro
from luna_cpp_b200.mesh import build_mesh, jittered_points
from luna_cpp_b200.problems import point_blast
from luna_cpp_b200.remesh import Remesher

pytestmark = pytest.mark.gpu

FIELDS = ("owner", "neighbour", "cell_face_start", "cell_face", "area", "face_centroid", "centroid", "volume", "positions")


# LUNA_MESH_DUAL=0 in the environment switches the host builder's 3D cells to face loops while the device keeps plane
# triples: the two then agree to round-off (the same faces and lists; areas, centroids and volumes to 1e-12), not bit for
# bit.
HOST_FACE_LOOPS = os.environ.get("LUNA_MESH_DUAL") == "0"


def assert_same_mesh(host, dev):
    assert (dev.n_cells, dev.n_faces, dev.inconsistent) == (host.n_cells, host.n_faces, host.inconsistent)
    for f in FIELDS:
        a, b = np.ascontiguousarray(getattr(host, f)), np.ascontiguousarray(getattr(dev, f))
        assert a.shape == b.shape, f
        if HOST_FACE_LOOPS and host.dim == 3 and a.dtype.kind == "f":
            assert np.max(np.abs(a - b)) <= 1e-12 * max(np.max(np.abs(a)), 1e-300), f
        else:
            assert a.tobytes() == b.tobytes(), f


def cases():
    rng = np.random.default_rng(7)
    yield "jittered 16^3", jittered_points((16, 16, 16), jitter=0.1, seed=1), (1.0, 1.0, 1.0)
    yield "uniform random 1500", rng.random((1500, 3)), (1.0, 1.0, 1.0)
    box = (1.0, 0.8, 1.2)
    yield "random, box 1 x 0.8 x 1.2", rng.random((1200, 3)) * np.array(box), box
    yield "jittered, outside the box", jittered_points((10, 10, 10), jitter=0.1, seed=3) + np.array([1.0, -2.0, 0.5]), (1.0, 1.0, 1.0)
    yield "2D jittered 40^2", jittered_points((40, 40), jitter=0.1, seed=1), (1.0, 1.0)
    yield "2D uniform random 2000", rng.random((2000, 2)), (1.0, 1.0)


@pytest.mark.parametrize("name,points,box", list(cases()), ids=[c[0] for c in cases()])
def test_device_mesh_equals_host_builder(cuda, name, points, box):
    host = build_mesh(points, box=box)
    r = Remesher(len(box), box)
    dev = r.build(points).to_host()
    assert_same_mesh(host, dev)
    voronoi_invariants(dev)
    r.close()


def test_remesher_reuse_grows_and_shrinks(cuda):
    """One remesher, meshes of different sizes in turn (its buffers are kept and grown)."""
    r = Remesher(3, (1.0, 1.0, 1.0))
    for nx in (8, 14, 6, 14):
        pts = jittered_points((nx,) * 3, jitter=0.1, seed=nx)
        assert_same_mesh(build_mesh(pts), r.build(pts).to_host())
    assert r.device_bytes() > 0
    r.close()


def test_remesher_errors_are_status_codes(cuda):
    r = Remesher(3, (1.0, 1.0, 1.0))
    with pytest.raises(hydro.LunaError) as e:  # two points: each cell reaches its own images
        r.build(np.array([[0.5, 0.5, 0.5], [0.1, 0.1, 0.1]]))
    assert e.value.status == 1
    pts = jittered_points((6, 6, 6), jitter=0.1, seed=1)
    pts[3, 1] = np.nan
    with pytest.raises(hydro.LunaError) as e:
        r.build(pts)
    assert e.value.status == 1
    # still usable after an error
    good = jittered_points((6, 6, 6), jitter=0.1, seed=1)
    assert_same_mesh(build_mesh(good), r.build(good).to_host())
    r.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32", "grad16"])
def test_static_step_on_device_tiles_equals_host_tiles(cuda, precision):
    """The same mesh given in host memory (tiles cut on the host, greedily) and in device memory (tiles cut on the
    device, fixed Morton chunks): five static steps give the same bits."""
    mesh = jittered_mesh(20)
    r = Remesher(3, mesh.box)
    dmesh = r.build(mesh.positions)
    q0 = point_blast(mesh)
    a = hydro.FiniteVolume(mesh, precision=precision)
    b = hydro.FiniteVolume(dmesh, precision=precision)
    a.set_state(q0)
    b.set_state(q0)
    for _ in range(5):
        dt = a.time_step(0.3)
        assert b.time_step(0.3) == dt
        a.step(dt)
        b.step(dt)
    assert np.array_equal(a.get_state(), b.get_state())
    assert np.array_equal(a.gradients(), b.gradients())
    a.close()
    b.close()
    r.close()


@pytest.mark.parametrize("dim", [3, 2])
def test_moving_step_with_device_remesh_equals_host_remesh(cuda, dim):
    """Moving steps (the t^n fluxes, the drift on the 2^-30 grid, the remesh, the t^n+1 fluxes) with the generators and
    the mesh kept on the device against the same steps with the host remesh: the same dt, positions and state, bit for
    bit; mass and energy conserved to round-off."""
    step = 2.0 ** -30
    nx = 12 if dim == 3 else 40
    pts = np.round(jittered_points((nx,) * dim, jitter=0.1, seed=1) / step) * step
    mesh = build_mesh(pts, box=(1.0,) * dim)
    q0 = point_blast(mesh, radius_cells=2.5)
    host = hydro.FiniteVolume(mesh, motion="moving")
    dev = hydro.FiniteVolume(mesh, motion="moving")
    host.set_state(q0)
    dev.set_state(q0)
    r = Remesher(dim, mesh.box)
    lib = hydro.lib()
    for _ in range(4):
        dt = host.time_step(0.3)
        assert dev.time_step(0.3) == dt
        mh = host.step_moving(dt, lambda p: build_mesh(p, box=(1.0,) * dim))
        # dev.step_moving_device(dt, r) in its three calls, the new mesh checked before the hydro takes it
        ptr = r.points_buffer(dev.n)
        hydro.check(lib.luna_fv_step_moving_begin(dev.handle, dt, ptr, 1))
        md = r.build_device(ptr, dev.n)
        assert_same_mesh(mh, md.to_host())
        hydro.check(lib.luna_fv_step_moving_end(dev.handle, ctypes.byref(md.desc)))
    dt = host.time_step(0.3)
    assert dev.time_step(0.3) == dt
    host.step_moving(dt, lambda p: build_mesh(p, box=(1.0,) * dim))
    dev.step_moving_device(dt, r)
    qh, qd = host.get_state(), dev.get_state()
    assert np.array_equal(qh, qd)
    assert abs(qd[:, 0].sum() - q0[:, 0].sum()) / q0[:, 0].sum() < 1e-14
    assert abs(qd[:, -1].sum() - q0[:, -1].sum()) / q0[:, -1].sum() < 1e-14
    host.close()
    dev.close()
    r.close()


def test_device_mesh_64cubed_equals_host_builder(cuda):
    """A 64^3 jittered mesh (262,144 cells, 2.1 M faces): the device build equals the host build."""
    pts = jittered_points((64, 64, 64), jitter=0.1, seed=1)
    r = Remesher(3, (1.0, 1.0, 1.0))
    assert_same_mesh(build_mesh(pts), r.build(pts).to_host())
    r.close()
