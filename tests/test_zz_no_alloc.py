"""The allocation-free flux-and-update pass (luna_apply_static_noalloc) through the C ABI, against the regular step
(luna_fv_step) on the same inputs, two calls in a row, within the one-step tolerance of the parity tests (1e-13 relative).

Callers of this entry point cannot allocate device memory themselves (a fixed device footprint, or a runtime that owns
every allocation); this test, which is not such a caller, allocates the inputs with torch. It sits in a file pytest
collects last, so a run that stops at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

from conftest import jittered_mesh
from luna_cpp_b200 import hydro
from luna_cpp_b200.problems import point_blast

pytestmark = pytest.mark.gpu

TOL = 1e-13


def device_desc(mesh, torch, keep):
    dev = torch.device("cuda")
    arrays = [torch.tensor(np.ascontiguousarray(a), device=dev) for a in (
        mesh.owner, mesh.neighbour, mesh.cell_face_start, mesh.cell_face, mesh.area, mesh.face_centroid, mesh.centroid,
        mesh.volume, mesh.positions)]
    keep.extend(arrays)
    d = hydro.MeshDesc()
    d.dim = mesh.dim
    d.n_cells = mesh.n_cells
    d.n_faces = mesh.n_faces
    (d.owner, d.neighbour, d.cell_face_start, d.cell_face, d.area, d.face_centroid, d.centroid, d.volume,
     d.positions) = [a.data_ptr() for a in arrays]
    for a in range(3):
        d.box[a] = mesh.box[a] if a < mesh.dim else 0.0
    d.on_device = 1
    return d


def padded(rows, width, torch):
    out = torch.zeros((rows.shape[0], width), dtype=torch.float64, device="cuda")
    out[:, : rows.shape[1]] = torch.tensor(rows, device="cuda")
    return out


@pytest.mark.parametrize("order", [1, 0])
def test_noalloc_pass_matches_the_step_twice(cuda, order):
    import torch

    mesh = jittered_mesh(16)
    q0 = point_blast(mesh, radius_cells=2.5)
    keep = []
    desc = device_desc(mesh, torch, keep)
    gas = hydro._Gas(5.0 / 3.0, 1e-10, 1e-10)
    fv = hydro.FiniteVolume(mesh, order=order)
    fv.set_state(q0)
    q = torch.tensor(q0, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        dt = fv.time_step(0.3)
        prims = padded(fv.prims(), 8, torch)
        grads = padded(fv.gradients(), 16, torch) if order == 1 else None
        fallbacks = ctypes.c_int64(-1)
        hydro.check(hydro.lib().luna_apply_static_noalloc(
            ctypes.byref(desc), ctypes.byref(gas), order, 0, ctypes.c_void_p(prims.data_ptr()),
            ctypes.c_void_p(grads.data_ptr() if grads is not None else 0), ctypes.c_void_p(q.data_ptr()), dt,
            ctypes.c_void_p(stream), ctypes.byref(fallbacks)))
        fv.step(dt)
        want = fv.get_state()
        got = q.cpu().numpy()
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < TOL, call
        assert fallbacks.value == fv.fallbacks()


def test_noalloc_rejects_meshes_beyond_its_scratch(cuda):
    """More faces than the fixed 32 MiB array holds: LUNA_EINVAL with a message, before any pointer is touched."""
    d = hydro.MeshDesc()
    d.dim = 3
    d.n_cells = 200000
    d.n_faces = 838855
    d.box[0] = d.box[1] = d.box[2] = 1.0
    d.on_device = 1
    d.owner = d.neighbour = d.cell_face_start = d.cell_face = d.area = d.face_centroid = d.centroid = 8
    d.volume = d.positions = 8
    gas = hydro._Gas(5.0 / 3.0, 1e-10, 1e-10)
    status = hydro.lib().luna_apply_static_noalloc(ctypes.byref(d), ctypes.byref(gas), 0, 0, None, None,
                                                   ctypes.c_void_p(8), 1e-3, None, None)
    assert status == 1
    assert b"838854" in hydro.lib().luna_last_error()


def test_noalloc_reports_a_state_that_is_not_finite(cuda):
    """A NaN planted in Q on the host: the update's error word comes back as LUNA_ENONFINITE when the call reads its
    counters (fallbacks_out given), as every other entry point reports it; the next clean call returns LUNA_OK."""
    import torch

    mesh = jittered_mesh(8)
    q0 = point_blast(mesh, radius_cells=2.0)
    keep = []
    desc = device_desc(mesh, torch, keep)
    gas = hydro._Gas(5.0 / 3.0, 1e-10, 1e-10)
    stream = torch.cuda.current_stream().cuda_stream
    bad = q0.copy()
    bad[5, 0] = np.nan
    for q_host, want in ((bad, 4), (q0, 0)):
        q = torch.tensor(q_host, device="cuda")
        fallbacks = ctypes.c_int64(-1)
        status = hydro.lib().luna_apply_static_noalloc(
            ctypes.byref(desc), ctypes.byref(gas), 0, 0, None, None, ctypes.c_void_p(q.data_ptr()), 1e-4,
            ctypes.c_void_p(stream), ctypes.byref(fallbacks))
        assert status == want, (status, hydro.lib().luna_last_error())
        if want == 4:
            assert b"not finite" in hydro.lib().luna_last_error()
