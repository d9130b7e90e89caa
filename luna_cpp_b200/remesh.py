"""The moving mesh's remesh on the device (include/luna_remesh.h), over ``libluna_b200.so``.

luna-cpp's ``FiniteVolume::move()`` (src/hydro/finite_volume.hpp:1212-1250) drifts the generators and has voronoi-cpp
update the mesh between the two flux passes of a moving step. ``Remesher`` rebuilds that mesh from the drifted
generators on the GPU, one thread per cell running the host builder's clipping code, so a ``DeviceMesh`` holds the same
arrays, bit for bit, as ``luna_cpp_b200.mesh.build_mesh`` gives for the same points; ``FiniteVolume.step_moving_device``
runs a whole moving step with the generators and the mesh kept on the device.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import hydro
from .mesh import Mesh


def _to_host(ptr: int, dtype, shape) -> np.ndarray:
    """A host copy of device memory (the CUDA runtime's cudaMemcpy through cuda-python)."""
    from cuda.bindings import runtime as rt

    out = np.empty(shape, dtype=dtype)
    if out.nbytes:
        (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        if err != rt.cudaError_t.cudaSuccess:
            raise RuntimeError(f"cudaMemcpy: {err}")
    return out


@dataclass
class CellArrays:
    dim: int
    box: tuple
    positions: np.ndarray
    centroid: np.ndarray
    volume: np.ndarray

    @property
    def n_cells(self) -> int:
        return int(self.volume.shape[0])


class DeviceMesh:
    """A mesh the remesher built: a ``luna_mesh_desc`` of device pointers (valid until the remesher's next build)."""

    def __init__(self, desc: hydro.MeshDesc, inconsistent: int):
        self.desc = desc
        self.dim = int(desc.dim)
        self.n_cells = int(desc.n_cells)
        self.n_faces = int(desc.n_faces)
        self.box = tuple(float(desc.box[a]) for a in range(self.dim))
        self.inconsistent = int(inconsistent)

    def cells(self):
        """Host copies of the per-cell arrays only (generators, centroids, volumes), for initial states and profiles."""
        d, N = self.dim, self.n_cells
        return CellArrays(dim=d, box=self.box, positions=_to_host(self.desc.positions, np.float64, (N, d)),
                          centroid=_to_host(self.desc.centroid, np.float64, (N, d)),
                          volume=_to_host(self.desc.volume, np.float64, (N,)))

    def to_host(self) -> Mesh:
        d, N, F = self.dim, self.n_cells, self.n_faces
        return Mesh(dim=d, owner=_to_host(self.desc.owner, np.int32, (F,)),
                    neighbour=_to_host(self.desc.neighbour, np.int32, (F,)),
                    cell_face_start=_to_host(self.desc.cell_face_start, np.int32, (N + 1,)),
                    cell_face=_to_host(self.desc.cell_face, np.int32, (2 * F,)),
                    area=_to_host(self.desc.area, np.float64, (F, d)),
                    face_centroid=_to_host(self.desc.face_centroid, np.float64, (F, d)),
                    centroid=_to_host(self.desc.centroid, np.float64, (N, d)),
                    volume=_to_host(self.desc.volume, np.float64, (N,)),
                    positions=_to_host(self.desc.positions, np.float64, (N, d)), box=self.box,
                    inconsistent=self.inconsistent)


class Remesher:
    """luna_remesh: periodic Voronoi meshes built on the GPU, in the box [0, box_a) per axis."""

    def __init__(self, dim: int = 3, box=(1.0, 1.0, 1.0)):
        self._h = ctypes.c_void_p()
        b = np.zeros(3, np.float64)
        b[: len(box)] = box
        self._box = b
        hydro.check(hydro.lib().luna_remesh_create(dim, b.ctypes.data, ctypes.byref(self._h)))
        self.dim = dim

    def points_buffer(self, n: int) -> int:
        """A device buffer of n x dim doubles owned by the remesher (luna_remesh_points)."""
        p = ctypes.c_void_p()
        hydro.check(hydro.lib().luna_remesh_points(self._h, n, ctypes.byref(p)))
        return int(p.value)

    def build(self, points) -> DeviceMesh:
        """The mesh of host points [n][dim]."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, self.dim)
        return self._build(pts.shape[0], pts.ctypes.data, 0)

    def build_device(self, ptr: int, n: int) -> DeviceMesh:
        """The mesh of n generators at the device pointer ptr."""
        return self._build(n, ptr, 1)

    def _build(self, n, ptr, on_device) -> DeviceMesh:
        desc = hydro.MeshDesc()
        inconsistent = ctypes.c_int64()
        hydro.check(hydro.lib().luna_remesh_build(self._h, n, ptr, on_device, ctypes.byref(desc), ctypes.byref(inconsistent)))
        return DeviceMesh(desc, inconsistent.value)

    def device_bytes(self) -> int:
        out = ctypes.c_int64()
        hydro.check(hydro.lib().luna_remesh_device_bytes(self._h, ctypes.byref(out)))
        return int(out.value)

    def close(self) -> None:
        if self._h:
            hydro.lib().luna_remesh_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
